"""Build hsolver_b200/libhsolver_b200.so in-tree with nvcc for sm_100a.

FMA contraction is off (-fmad=false) so every point update rounds like the
reference's scalar x86-64 arithmetic; division and square root stay IEEE.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhsolver_b200.so")
SOURCES = ["hs_case.cpp", "hs_api.cpp", "hs_engine.cu", "hs_cht.cu", "hs_channel.cu", "hs_slab.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-v"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def build(verbose=False):
    """Compile every source and link the shared library; returns its path."""
    objs = []
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(bdir, src + ".o")
        path = os.path.join(CSRC, src)
        deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".hpp", ".cuh"))]
        deps.append(os.path.join(os.path.dirname(HERE), "include", "hsolver_b200.h"))
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(d) for d in deps):
            cmd = [_nvcc()] + ARCH + NVCC_FLAGS + ["-c", path, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [_nvcc(), "-x", "cu"] + ARCH + NVCC_FLAGS + ["-c", path, "-o", obj]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("nvcc failed on %s" % src)
            if verbose:
                sys.stderr.write(r.stderr)
        objs.append(obj)
    cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
