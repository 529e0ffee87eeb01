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


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


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
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force or a.verbose))
