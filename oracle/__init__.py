"""Parity oracle (TEST INFRASTRUCTURE ONLY).

  oracle/_ref/libvlrref.so   built by oracle/build_ref.sh: the reference's own
                             spectral code (libVLR/shared) and BSDF/EDF classes
                             (GPU_kernels/materials.cu) compiled for the host,
                             FP32 as shipped, plus ref_shim.cpp, which exposes
                             them and holds the CPU restatements of the
                             reference's integrators built on them:
                               ref_pt.inc   path_tracing.cu (camera, closest
                                            hit, NEE, MIS, the environment's
                                            miss program and importance maps;
                                            point emitters, a Matte albedo
                                            texture and a normal map on demand)
                               ref_bpt.inc  lvc_bpt.cu (light vertex cache,
                                            connections, MIS recursion);
  oracle/_build/liboracle.so our sequential restatement of the LBVH build and
                             the treelet restructuring pass (lbvh_host.c);
  ref.py / lbvh.py           ctypes bindings of the two libraries;
  guide_ref.py               numpy model of the guiding network (BF16-rounded
                             forward, analytic backward).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg and
reference arm use this package; the product library never links, loads or
calls it.
"""
