"""Build the sm_100a shared library of the hot path in-tree.

    python -m lbcuda_b200.build          # -> lbcuda_b200/liblbx.so

The library is plain nvcc output (no torch extension): its C ABI is
include/lbx.h, loaded from Python through ctypes.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblbx.so")
DRIVER = os.path.join(HERE, "lbx_run")

SOURCES = ["lbx_api.cu", "lbx_fluid.cu", "lbx_fused.cu", "lbx_particles.cu", "lbx_closure.cu", "lbx_ensemble.cu",
           "lbx_noalloc.cu"]
HOST_SOURCES = ["lbx_driver.cpp"]
OBJDIR = os.path.join(HERE, "_build")
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC",
    "-I", os.path.join(ROOT, "include"),
]
# The single-pass fluid kernels write every fused multiply-add explicitly and
# are compiled without contraction, so each kernel that inlines them (one box,
# particle box, ensemble) performs the same roundings.  The BGK and two-pass
# kernels follow the reference's expression order and are compiled without
# contraction as well, so they round as the reference's FP32 arithmetic does.
FILE_FLAGS = {"lbx_fused.cu": ["-fmad=false"], "lbx_fluid.cu": ["-fmad=false"]}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def build(verbose=False, extra=()):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(CSRC, h) for h in os.listdir(CSRC)]
                 + [os.path.join(ROOT, "include", "lbx.h"), os.path.abspath(__file__)])
    fresh = all(os.path.exists(f) and os.path.getmtime(f) >= newest for f in (LIB, DRIVER))
    if fresh and not extra:
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    objs = [os.path.join(OBJDIR, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    cmds = [[nvcc()] + NVCC_FLAGS + FILE_FLAGS.get(s, []) + list(extra) + ["-c", src, "-o", obj]
            for s, src, obj in zip(SOURCES, srcs, objs)]
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        procs = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for c, p in zip(cmds, procs):
        if verbose or p.returncode:
            print(" ".join(c), flush=True)
            sys.stdout.write(p.stdout)
            sys.stderr.write(p.stderr)
        if p.returncode:
            raise subprocess.CalledProcessError(p.returncode, c)
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared"] + objs + ["-o", LIB]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    # command-line host (input.dat driver), linked against the library
    cmd = ["g++", "-O2", "-std=c++17", os.path.join(CSRC, "lbx_driver.cpp"), "-I", os.path.join(ROOT, "include"),
           "-I", "/usr/local/cuda/include", "-L", HERE, "-llbx", "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath,$ORIGIN", "-Wl,-rpath,/usr/local/cuda/lib64", "-o", DRIVER]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
