"""Builds libllb200.so in-tree (cudalucas_b200/libllb200.so) with nvcc for
sm_100a.  Usage: python -m cudalucas_b200.build [--debug]"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libllb200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["engine.cu", "host_util.cpp"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(verbose=False, extra=()):
    srcs = [os.path.join(SRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(SRC, h) for h in os.listdir(SRC) if h.endswith(".cuh")] + [os.path.join(ROOT, "include", "llb200.h")]
    if os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in deps) and not extra:
        return OUT
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-I", os.path.join(ROOT, "include"), *extra, "-o", OUT + ".tmp", *srcs, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


CLI_SRC = os.path.join(HERE, "host", "llucas.cpp")
CLI_OUT = os.path.join(HERE, "bin", "llucas")


def build_cli(verbose=False):
    """The command-line tester (C++ host over the C ABI), linked to the
    in-tree libllb200.so through an $ORIGIN-relative rpath."""
    build()
    deps = [CLI_SRC, os.path.join(ROOT, "include", "llb200.h"), OUT]
    if os.path.exists(CLI_OUT) and all(os.path.getmtime(CLI_OUT) >= os.path.getmtime(d) for d in deps):
        return CLI_OUT
    os.makedirs(os.path.dirname(CLI_OUT), exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), "-o", CLI_OUT + ".tmp",
           CLI_SRC, "-L", HERE, "-lllb200", "-Wl,-rpath,$ORIGIN/.."]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(CLI_OUT + ".tmp", CLI_OUT)
    return CLI_OUT


if __name__ == "__main__":
    extra = []
    if "--ptxas-v" in sys.argv:
        extra += ["-Xptxas", "-v"]
    print(build(verbose=True, extra=extra))
    print(build_cli(verbose=True))
