"""Build recipe for the in-tree CUDA library ds2d_b200/libds2d_b200.so (sm_100a only)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libds2d_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "ds2d_engine.cu"), os.path.join(HERE, "csrc", "ds2d_unet.cu")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))] + [
    os.path.join(ROOT, "include", "ds2d.h")]
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared"]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in DEPS if os.path.exists(p))


HOST_MAIN = os.path.join(HERE, "csrc", "host", "ds2d_main.cpp")
HOST_BIN = os.path.join(HERE, "ds2d_elsrtm")


def build(force=False, verbose=False):
    if force or stale():
        cmd = [_nvcc()] + NVCC_FLAGS + ["-o", LIB] + SOURCES
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(HOST_BIN) or os.path.getmtime(HOST_BIN) < max(
            os.path.getmtime(LIB), os.path.getmtime(HOST_MAIN)):
        # C++ host driver (parameters file, SU I/O, shot loop) linked against the library.
        cmd = ["g++", "-O2", "-std=c++17", "-o", HOST_BIN, HOST_MAIN, "-L" + HERE, "-lds2d_b200",
               "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
