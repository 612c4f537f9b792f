"""Build liblinqt_gpu.so in-tree with nvcc for sm_100a, and liblinqt_facade.so.

    python -m linqt_b200.build          # or linqt_b200.build.build()

The GPU library is compiled from linqt_b200/csrc/*.cu with the CUDA runtime linked
statically, so the .so carries no dependency on a particular libcudart.  The facade
library (linqt_b200/facade: LinQT's C++ classes on the C ABI) and the wannier2sparse
command line (linqt_b200/w2s) are plain C++ linked against it.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblinqt_gpu.so")
FACADE = os.path.join(HERE, "facade")
FACADE_LIB = os.path.join(HERE, "liblinqt_facade.so")
W2S_SRC = os.path.join(HERE, "w2s", "wannier2sparse.cpp")
W2S_BIN = os.path.join(HERE, "w2s", "_bin", "wannier2sparse")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
         "-diag-suppress", "177"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "linqt_gpu.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build_facade(force=False, verbose=False):
    srcs = glob.glob(os.path.join(FACADE, "*.cpp"))
    deps = srcs + glob.glob(os.path.join(FACADE, "include", "*.hpp")) + [LIB, os.path.join(ROOT, "include", "linqt_gpu.h")]
    if not force and os.path.exists(FACADE_LIB) and all(os.path.getmtime(p) <= os.path.getmtime(FACADE_LIB)
                                                        for p in deps):
        return FACADE_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", os.path.join(FACADE, "include"), "-I",
           os.path.join(ROOT, "include"), "-o", FACADE_LIB] + srcs + ["-L", HERE, "-llinqt_gpu",
                                                                      "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("g++ (facade) failed:\n" + p.stdout + p.stderr)
    return FACADE_LIB


def build_w2s(force=False, verbose=False):
    """The wannier2sparse command line on liblinqt_gpu.so (linqt_b200/w2s/_bin/wannier2sparse)."""
    deps = [W2S_SRC, LIB, os.path.join(ROOT, "include", "linqt_gpu.h")]
    if not force and os.path.exists(W2S_BIN) and all(os.path.getmtime(p) <= os.path.getmtime(W2S_BIN) for p in deps):
        return W2S_BIN
    os.makedirs(os.path.dirname(W2S_BIN), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-o", W2S_BIN, W2S_SRC, "-L", HERE,
           "-llinqt_gpu", "-Wl,-rpath,$ORIGIN/../.."]
    if verbose:
        print(" ".join(cmd))
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("g++ (wannier2sparse) failed:\n" + p.stdout + p.stderr)
    return W2S_BIN


def build(force=False, verbose=False, extra=()):
    if force or needs_build():
        cmd = [nvcc()] + ARCH + FLAGS + list(extra) + ["-I", os.path.join(ROOT, "include"), "-o", LIB] + sources()
        if verbose:
            print(" ".join(cmd))
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + p.stdout + p.stderr)
    build_facade(force=force, verbose=verbose)
    build_w2s(force=force, verbose=verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
