"""Build liblgv.so (the CUDA library behind include/lgv.h) in-tree.

    python langevina_b200/build.py [--verbose]

Compiles every .cu under langevina_b200/csrc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) into langevina_b200/liblgv.so.
nvcc cross-compiles without a GPU.
"""
import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "liblgv.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


DRIVER = os.path.join(HERE, "superpions")
CXX = os.environ.get("CXX", "g++")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def build_driver():
    """The C++ run driver (csrc/superpions.cpp) over include/langevina.hpp, linked to liblgv.so."""
    src = os.path.join(HERE, "csrc", "superpions.cpp")
    deps = [src, LIB, os.path.join(REPO, "include", "langevina.hpp"), os.path.join(REPO, "include", "lgv.h")]
    if os.path.exists(DRIVER) and all(os.path.getmtime(d) <= os.path.getmtime(DRIVER) for d in deps):
        return DRIVER
    cmd = [CXX, "-O2", "-std=c++17", "-Wall", "-I", os.path.join(REPO, "include"), src, "-o", DRIVER,
           "-L", HERE, "-llgv", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("g++ failed building the superpions driver")
    return DRIVER


def headers():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh"))
                  + glob.glob(os.path.join(REPO, "include", "*.h")))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [__file__])


def build(verbose=False, force=False):
    if not force and up_to_date():
        build_driver()
        return LIB
    cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "--shared", "-Xcompiler", "-fPIC",
           "-I", os.path.join(REPO, "include"), "-o", LIB, *sources()]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building liblgv.so")
    if verbose:
        sys.stderr.write(r.stderr)
    build_driver()
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force or a.verbose))
