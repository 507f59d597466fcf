"""Build the engine library in-tree (sirius_b200/libsirius_b200.so) for sm_100a.

nvcc cross-compiles without a GPU. The .so is git-ignored but travels with the
repository snapshot to the GPU host.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
LIB = os.path.join(HERE, "libsirius_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def sources():
    srcs = [os.path.join(CSRC, "engine.cu")]
    if os.path.isdir(HOST):
        srcs += sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp"))
    return srcs


def _deps():
    files = []
    for d in (CSRC, HOST, os.path.join(ROOT, "include")):
        if os.path.isdir(d):
            files += [os.path.join(d, f) for f in os.listdir(d)]
    return files


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-shared", "-o", LIB + ".tmp", *sources(), "-lz"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
