"""Builds libicoadv.so in-tree with nvcc for sm_100a.

Each CUDA source is compiled with its own flags (the plain reference-interface
kernels without FMA contraction, so their FP64 arithmetic is the reference's
operation sequence) and linked into one shared library next to this file.
Rebuilds only when a source or header is newer than the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libicoadv.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          f"-I{INCLUDE}", f"-I{CSRC}"]

# source -> extra flags
SOURCES = {
    "topology.cpp": [],
    "capi.cu": [],
    "plain_kernels.cu": ["--fmad=false"],
    "step.cu": ["--fmad=false"],
    "fast_kernels.cu": [],
    "noalloc.cu": [],
    "adjoint.cu": ["--fmad=false"],
    "geometry.cu": ["--fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libicoadv")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    objs = []
    cc = nvcc()
    for src, extra in SOURCES.items():
        path = CSRC / src
        if not path.exists():
            continue
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if _stale(obj, [path, *headers, Path(__file__)]):
            cmd = [cc, *ARCH, *COMMON, *extra, "-c", str(path), "-o", str(obj)]
            if src.endswith(".cpp"):
                cmd = [shutil.which("g++") or "g++", "-O3", "-std=c++17", "-fPIC", "-Wall",
                       f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(path), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [cc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
