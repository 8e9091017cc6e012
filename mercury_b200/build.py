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
                                               "mb_voxel.cpp", "mb_noalloc.cu", "mb_devo.cu", "mb_voxel_dev.cu", "mb_surrogate.cu", "mb_knn.cu", "mb_probe.cu")]
DEPS = SRC + [os.path.join(HERE, "csrc", f) for f in ("mb_internal.h", "mb_sin.cuh", "mb_pack.h", "mb_devo.h", "mb_voxel.h", "mb_voxel_dev.h", "mb_sg_kernels.cuh")] + [
    os.path.join(ROOT, "include", "mercury_b200.h")]
OUT = os.path.join(HERE, "libmercury_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
          "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "-Xcompiler", "-fvisibility=hidden"]
OBJ_DIR = os.path.join(HERE, "_build")


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in DEPS)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object in parallel (mercury_b200/_build),
    then links libmercury_b200.so."""
    if force or not up_to_date():
        from concurrent.futures import ThreadPoolExecutor
        os.makedirs(OBJ_DIR, exist_ok=True)
        objs = [os.path.join(OBJ_DIR, os.path.basename(src) + ".o") for src in SRC]
        extra = ["-Xptxas=-v"] if verbose else []
        with ThreadPoolExecutor(max_workers=len(SRC)) as ex:
            logs = list(ex.map(lambda so: _run([NVCC, *COMMON, *extra, "-c", "-o", so[1], so[0]]),
                               zip(SRC, objs)))
        _run([NVCC, *COMMON, "-shared", "-o", OUT, *objs, "-lpthread"])
        if verbose:
            print("\n".join(logs))
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
