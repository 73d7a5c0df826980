"""Build libmslice_b200.so in-tree with nvcc for sm_100a.

Usage: ``python -m cudamultislice_b200.build [--force]``.  Objects go to
``cudamultislice_b200/_build/``; the shared library lands next to this file
so that it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmslice_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["ms_engine.cu", "ms_slice.cu", "ms_atoms.cu", "ms_pointwise.cu", "ms_noalloc.cu", "ms_tiff.cu",
           "ms_slice_n64.cu", "ms_slice_n128.cu", "ms_slice_n256.cu", "ms_slice_n512.cu", "ms_slice_n1024.cu",
           "ms_slice_n2048.cu", "ms_slice_n4096.cu", "ms_slice_loop.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", f"-I{INCLUDE}"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_lib_dir(nvcc: str) -> str:
    return os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "lib64")


def _deps() -> list[str]:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, "mslice.h"))
    files.append(os.path.abspath(__file__))
    return files


def _compile(nvcc: str, src: str) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = True) -> str:
    """Compile every CUDA source and link the shared library; returns its path."""
    newest = max(os.path.getmtime(f) for f in _deps())
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    if verbose:
        print(f"[cudamultislice_b200] building {os.path.basename(LIB)} for sm_100a", file=sys.stderr)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(nvcc, s), SOURCES))
    libdir = _cuda_lib_dir(nvcc)
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, f"-L{libdir}", "-lcufft",
           "-Xlinker", f"-rpath,{libdir}"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
