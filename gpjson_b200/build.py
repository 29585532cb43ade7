"""Ahead-of-time build of the native library for sm_100a.

The reference compiles its kernels at run time with NVRTC and no arch flag
(gpu/CUDARuntime.java:267-289); this package ships them compiled with nvcc
for sm_100a into ``gpjson_b200/_native/libgpjson_b200.so`` next to the
Python sources, so the built library travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
NATIVE = PKG / "_native"
LIB = NATIVE / "libgpjson_b200.so"
DATAGEN_SRC = PKG / "datagen" / "ndjson_gen.c"
DATAGEN_LIB = NATIVE / "libgpjson_datagen.so"
INCLUDE = PKG.parent / "include"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH_FLAGS + [
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC,-O3,-fvisibility=hidden",
    "-shared",
    "-cudart=static",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build gpjson_b200")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_native(force: bool = False, verbose: bool = False) -> Path:
    """Compiles libgpjson_b200.so if any source changed; returns its path."""
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "gpjson_b200.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    NATIVE.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), *NVCC_FLAGS, "-o", str(tmp), *map(str, sources())]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


def build_datagen(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the synthetic NDJSON generator (host code, OpenMP)."""
    if not force and not _stale(DATAGEN_LIB, [DATAGEN_SRC]):
        return DATAGEN_LIB
    NATIVE.mkdir(exist_ok=True)
    tmp = DATAGEN_LIB.with_suffix(".so.tmp")
    cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-fvisibility=hidden", "-o", str(tmp), str(DATAGEN_SRC), "-lm"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    tmp.replace(DATAGEN_LIB)
    return DATAGEN_LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_native(force, verbose)
    build_datagen(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
