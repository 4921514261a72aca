"""Build libvlr_b200.so in-tree with nvcc for sm_100a.

    python -m vlr_b200.build [--force]

Steps: (1) regenerate the spectral data tables from the reference sources when
the reference tree is available (otherwise an existing generated file is
reused); (2) compile every csrc/*.cu to an object with nvcc; (3) link the
shared library next to this file.  A translation unit is recompiled when it or
any csrc header is newer than its object.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvlr_b200.so")
GEN = os.path.join(CSRC, "generated", "spectral_tables.inc")
REFERENCE = os.environ.get("VLR_REFERENCE", "/root/reference")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = os.environ.get("VLR_HOST_CXX", "/usr/bin/g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-ccbin", HOST_CXX,
                 "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills",
                 "--expt-relaxed-constexpr", "-I", CSRC,
                 "-I", os.path.join(HERE, "..", "include")]
# Translation units whose results are compared query-by-query with the
# reference's host build: no FMA contraction.
NO_FMA = {"bsdf_batch.cu"}


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def generate_tables(force=False):
    if os.path.isdir(os.path.join(REFERENCE, "libVLR", "shared")):
        if force or not os.path.exists(GEN):
            subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_tables.py"), REFERENCE, GEN])
    elif not os.path.exists(GEN):
        raise RuntimeError(
            "spectral tables missing: %s does not exist and the reference tree (%s) is not "
            "available to generate it" % (GEN, REFERENCE))


def _compile(src, force):
    name = os.path.basename(src)
    obj = os.path.join(OBJ, name + ".o")
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + [GEN]
    headers += glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    headers += glob.glob(os.path.join(HERE, "..", "include", "vlr", "*.h"))
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _newest([src] + headers):
        return obj, None
    cmd = [NVCC] + COMMON + (["-fmad=false"] if name in NO_FMA else []) + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return obj, "%s\n%s\n%s" % (" ".join(cmd), p.stdout, p.stderr)
    return obj, None


def build(force=False, verbose=True):
    os.makedirs(OBJ, exist_ok=True)
    generate_tables(force=force)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, force), sources))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-o", LIB] + objs
        subprocess.check_call(cmd)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
