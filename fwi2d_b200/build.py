"""In-tree build of libfwi2d_b200.so for sm_100a.

The library is compiled with ``--fmad=false``: the kernels restate the
reference's single-precision operation order, and a contracted multiply-add
would round differently from the reference's CPU build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfwi2d_b200.so")
SOURCES = ["kernels.cu", "engine.cu", "noalloc.cu", "host_tables.cpp"]
HEADERS = ["engine.h", "launch.h", "sbp.cuh", "march.cuh", "zband.cuh", "xband.cuh", "acoustic.cuh", "resample.cuh", "host_tables.h",
           "d2_closure.inc", "../../include/fwi2d_b200.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
]
OBJDIR = os.path.join(HERE, "_build")

def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in SOURCES + HEADERS:
        p = os.path.join(CSRC, f)
        if os.path.exists(p) and os.path.getmtime(p) > t:
            return True
    return False


def build(force=False, verbose=False):
    """Compile every translation unit to an object in parallel (they share no
    device symbols), then link the shared library."""
    if not force and not stale():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    objs, procs = [], []
    for s in srcs:
        o = os.path.join(OBJDIR, os.path.splitext(s)[0] + ".o")
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", "-o", o, os.path.join(CSRC, s)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((s, subprocess.Popen(cmd, cwd=CSRC)))
        objs.append(o)
    failed = [s for s, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc " + " ".join(failed))
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp"] + objs
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
