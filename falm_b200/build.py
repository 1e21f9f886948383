"""Build the in-tree CUDA library falm_b200/libfalm_b200.so for sm_100a.

Run as ``python -m falm_b200.build``; __graft_entry__.build() calls build().
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = [os.path.join(HERE, "csrc", "falm_b200.cu")]
HEADERS = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh")))
OUT = os.path.join(HERE, "libfalm_b200.so")
NVCC_FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared"]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = SOURCES + HEADERS + [os.path.join(ROOT, "include", "falm_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


DRIVER_SRC = os.path.join(HERE, "csrc", "nedo_driver.cpp")
DRIVER = os.path.join(HERE, "nedo_driver")


def build(force=False, verbose=True):
    nvcc = os.environ.get("NVCC", "nvcc")
    if force or _stale():
        cmd = [nvcc] + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-o", OUT] + SOURCES
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    hpp = os.path.join(ROOT, "include", "falm_b200.hpp")
    if force or not os.path.exists(DRIVER) or max(os.path.getmtime(DRIVER_SRC), os.path.getmtime(hpp),
                                                   os.path.getmtime(OUT)) > os.path.getmtime(DRIVER):
        # the C++ driver over the class shim (include/falm_b200.hpp), linked to the library
        cmd = [nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-x", "cu", "-I", os.path.join(ROOT, "include"), DRIVER_SRC, "-o", DRIVER,
               "-L", HERE, "-lfalm_b200", "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
