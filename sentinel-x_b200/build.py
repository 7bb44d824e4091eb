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
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
# the kernel instantiations sit in their own translation units so they
# compile in parallel
SOURCES = ["engine.cu", "pack.cu", "scheduler.cu", "domain_passes.cu", "score.cu", "static_entry.cu", "k_msv.cu",
           "k_msv16.cu", "k_vit16.cu", "k_vit.cu", "k_vbin.cu", "k_env.cu", "hmmfile.cpp", "domains.cpp"]
HEADERS = ["engine.hpp", "kernels.cuh", "adjoint.cuh", "plain.cuh", "long.cuh", "envelope.cuh", "internal.hpp", "shapes.hpp", "prescreen.cuh",
           "tuned_shapes.inc"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def common():
    return [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
            "-Xptxas", "-v" if os.environ.get("SX_PTXAS_VERBOSE") else "-O3",
            "-Xcompiler", "-fPIC,-O3,-ffp-contract=off,-fno-fast-math", "-I", INCLUDE]


def obj_of(src):
    return os.path.join(OBJ, os.path.splitext(src)[0] + ".o")


def compile_cmd(src):
    return common() + ["-c", os.path.join(CSRC, src), "-o", obj_of(src)]


def link_cmd():
    # only the C ABI is exported (csrc/exports.map)
    return common() + ["-shared", "-o", OUT] + [obj_of(s) for s in SOURCES] + [
        "-Xlinker", "--version-script=" + os.path.join(CSRC, "exports.map"), "-lz", "-lpthread"]


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS + ["exports.map"]] + [os.path.join(INCLUDE, "sxhmm.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def _run(c):
    r = subprocess.run(c, capture_output=True, text=True)
    return r.returncode, r.stdout + r.stderr


def build(force=False):
    if not force and not stale():
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        results = list(ex.map(_run, [compile_cmd(s) for s in SOURCES]))
    for src, (rc, out) in zip(SOURCES, results):
        if rc != 0 or os.environ.get("SX_PTXAS_VERBOSE"):
            sys.stderr.write(out)
        if rc != 0:
            raise RuntimeError(f"nvcc failed compiling {src}")
    rc, out = _run(link_cmd())
    if rc != 0:
        sys.stderr.write(out)
        raise RuntimeError("nvcc failed linking libsxhmm.so")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
