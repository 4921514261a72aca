"""Parity oracle (TEST INFRASTRUCTURE ONLY).

  oracle/_ref/libvlrref.so   the reference's own spectral + BSDF code built for
                             the host by oracle/build_ref.sh (FP32, as shipped);
  oracle/_build/libvlroracle.so
                             our CPU restatement of the reference's algorithms
                             (oracle/vlr_oracle.cpp) in FP32 and FP64, including
                             the path-tracing and LVC-BPT integrators.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package; the product library never links, loads or calls it.
"""
