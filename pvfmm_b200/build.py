"""Builds libpvfmm_b200.so in-tree with nvcc for sm_100a (B200).

Run ``python -m pvfmm_b200.build`` (or ``__graft_entry__.build()``).  Objects
are cached under ``pvfmm_b200/_build`` and rebuilt when a source or header is
newer than its object.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libpvfmm_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--extended-lambda", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-fopenmp,-O3", f"-I{ROOT / 'include'}", f"-I{CSRC}"]
SOURCES = ["precomp.cpp", "tree.cu", "eval.cu", "hadamard_tc.cu", "translate.cu", "capi.cu", "direct.cu"]


def _newer(src: Path, obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, extra_flags=None) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    objs = []
    flags = CUDA_FLAGS + (extra_flags or [])
    for name in SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        objs.append(obj)
        if not _newer(src, obj, headers):
            continue
        cmd = [NVCC] + ARCH + flags + ["-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd = [os.environ.get("CXX", "g++"), "-O3", "-std=c++17", "-fPIC", "-fopenmp",
                   f"-I{ROOT / 'include'}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + \
              ["-lgomp", "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
