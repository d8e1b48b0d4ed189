"""Build the native library in-tree.

    python sabertooth_b200/_build.py          # libsabertooth_b200.so for sm_100a

nvcc compiles the CUDA runtime, the kernels (sm_100a, B200) and the serving
loops into one shared library next to this file, so the built .so travels with
the source tree.  Rebuilds only when a source is newer than the library.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libsabertooth_b200.so")

SOURCES = ["st_runtime.cu", "st_noalloc.cu", "st_server.cpp"]
HEADERS = ["st_common.cuh", "st_sw16.cuh", "st_sw32.cuh", "st_ungapped.cuh", "st_tuning.h", "st_dplan.cuh", "st_gate.cuh", "st_calib.cuh", "st_seed.cuh"]
INCLUDES = [os.path.join(ROOT, "include", "sabertooth_b200.h")]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force=False, verbose=False):
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + INCLUDES
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [
        nvcc(),
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-lineinfo", "-O3", "-std=c++17",
        "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off",
        "-Xptxas", "-v" if verbose else "-O3",
        "-shared",
        "-o", LIB,
    ] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lgomp"]
    tmp = LIB + ".tmp"
    cmd[cmd.index("-o") + 1] = tmp
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libsabertooth_b200.so")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose="-v" in sys.argv))
