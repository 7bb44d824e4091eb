"""Build libsxhmm.so (the sm_100a engine) in-tree with nvcc.

    python sentinel-x_b200/build.py [--force]

Device code: -gencode arch=compute_100a,code=sm_100a, -fmad=false (the
kernels use explicit __fadd_rn/__fmul_rn as well) and -lineinfo for ncu.
Host code: -O3 -ffp-contract=off, because the host half of the pipeline
(domain definition) must round exactly like the reference, which never fuses
a*b+c.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "sxhmm", "libsxhmm.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
SOURCES = ["engine.cu", "hmmfile.cpp", "domains.cpp"]
HEADERS = ["kernels.cuh", "adjoint.cuh", "plain.cuh", "long.cuh", "envelope.cuh", "internal.hpp", "tuned_shapes.inc"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def cmd():
    return [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
            "-Xptxas", "-v" if os.environ.get("SX_PTXAS_VERBOSE") else "-O3",
            "-Xcompiler", "-fPIC,-O3,-ffp-contract=off,-fno-fast-math", "-shared", "-I", INCLUDE,
            "-o", OUT] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lz", "-lpthread"]


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "sxhmm.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False):
    if not force and not stale():
        return OUT
    c = cmd()
    r = subprocess.run(c, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libsxhmm.so")
    if os.environ.get("SX_PTXAS_VERBOSE"):
        sys.stderr.write(r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
