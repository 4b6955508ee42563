"""Builds libnsx.so (the CUDA hot path and its C ABI) in-tree for sm_100a.

    python -m nushellx_b200.build

nvcc compiles every .cu/.cpp under nushellx_b200/csrc with
``-gencode arch=compute_100a,code=sm_100a`` and links one shared library next
to this file.  Rebuilds only when a source or header is newer than the library.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libnsx.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         "-I", INCLUDE, "-I", CSRC]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    srcs = sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "nsx.h"))
    if not force and not _stale(LIB, srcs + headers):
        if _stale(CLI, [CLI_SRC, LIB]):
            build_cli(verbose)
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-c", s, "-o", o]
        if s.endswith(".cpp"):
            cmd.insert(1, "-x")
            cmd.insert(2, "cu")
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(o)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-lpthread", "-ldl", "-lrt"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    build_cli(verbose)
    return LIB


CLI_SRC = os.path.join(HERE, "cli", "nulnz_gpu.cpp")
CLI = os.path.join(HERE, "nulnz_gpu")


def build_cli(verbose=False):
    """The nulnz_gpu command (C++ host over the C ABI), linked against libnsx.so."""
    cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, CLI_SRC, "-o", CLI, "-L", HERE, "-lnsx",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return CLI


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
