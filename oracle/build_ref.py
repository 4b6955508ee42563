"""Builds oracle/libnsxref.so: the C/OpenMP restatement of the reference hot path
(test infrastructure; the timed host-core baseline).  gcc only, no GPU code."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "nsx_ref.c")
LIB = os.path.join(HERE, "libnsxref.so")


HEADER = os.path.join(ROOT, "include", "nsx.h")   # the problem structs it reads


def build(force=False):
    newest = max(os.path.getmtime(SRC), os.path.getmtime(HEADER))
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    # x86-64-v3 (AVX2/FMA): portable across the build host and the GPU hosts' CPUs
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c11",
           "-I", os.path.join(ROOT, "include"), SRC, "-o", LIB, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
