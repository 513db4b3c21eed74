"""Build step: compile the CUDA engine into ``libglst_b200.so`` (in place).

    python build.py            # or glst_b200.build.build()

nvcc cross-compiles for sm_100a without a GPU.  The shared library is written
next to this file, where the ctypes loader looks for it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libglst_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "engine.cu"), os.path.join(HERE, "csrc", "planner.cpp"),
           os.path.join(HERE, "csrc", "noalloc.cu")]
HEADERS = [os.path.join(HERE, "csrc", "kernels.cuh"), os.path.join(HERE, "csrc", "planner.hpp"),
           os.path.join(ROOT, "include", "glst_c.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.exists(c) or c == "nvcc"):
            return c
    return "nvcc"


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in SOURCES + HEADERS)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-shared",
           "-I" + os.path.join(ROOT, "include"), "-o", LIB + ".tmp", *SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
