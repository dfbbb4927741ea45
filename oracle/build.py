"""Build the CPU oracle (test infrastructure): oracle/liblbx_oracle.so.

    python -m oracle.build

Flags: -O3 with OpenMP; -ffp-contract=off keeps the reference's separate
multiply and add roundings; -march=x86-64-v3 (AVX2) so the library built
here also runs on the GPU hosts.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "lbx_oracle.cpp")
LIB = os.path.join(HERE, "liblbx_oracle.so")
FLAGS = ["-O3", "-fopenmp", "-fPIC", "-shared", "-std=c++17", "-ffp-contract=off",
         "-march=x86-64-v3", "-I", os.path.join(ROOT, "include")]


def build(verbose=False):
    deps = [SRC, os.path.join(ROOT, "include", "lbx.h")]
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        return LIB
    cmd = ["g++"] + FLAGS + [SRC, "-o", LIB]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
