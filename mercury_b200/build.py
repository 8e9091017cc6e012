"""Builds libmercury_b200.so in-tree for sm_100a with nvcc.

    python mercury_b200/build.py [--force] [-v]

(Run as a file: importing the package loads the library this builds.)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = [os.path.join(HERE, "csrc", f) for f in ("mb_kernels.cu", "mb_host.cpp", "mb_pack.cpp",
                                               "mb_voxel.cpp", "mb_noalloc.cu", "mb_devo.cu", "mb_voxel_dev.cu")]
DEPS = SRC + [os.path.join(HERE, "csrc", f) for f in ("mb_internal.h", "mb_sin.cuh", "mb_pack.h", "mb_devo.h", "mb_voxel.h", "mb_voxel_dev.h")] + [
    os.path.join(ROOT, "include", "mercury_b200.h")]
OUT = os.path.join(HERE, "libmercury_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "-Xcompiler", "-fvisibility=hidden", "-shared", "-lpthread"]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    if force or not up_to_date():
        cmd = [NVCC, *FLAGS, "-o", OUT, *SRC]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print(r.stderr)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
