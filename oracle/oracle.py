"""TEST INFRASTRUCTURE ONLY: numpy/ctypes front end of the C oracle
(gpjson_oracle.c) and of the Python JSONPath compiler restatement
(jsonpath_oracle.py).  Used by tests/, __graft_entry__.smoke() and the CPU
baseline legs of bench.py; never by the gpjson_b200 package.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import c_int, c_int64, c_void_p
from pathlib import Path

import numpy as np

from . import jsonpath_oracle

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_lib = None


def build(force: bool = False) -> Path:
    src = [HERE / "gpjson_oracle.c", HERE / "gpjson_oracle.h"]
    if force or not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in src):
        subprocess.run(["make", "-s", "-C", str(HERE), "-B" if force else "liboracle.so"], check=True)
    return LIB_PATH


# The reference checkout whose CUDA kernels oracle/_ref is built from
# (ref_gpu_driver.cu) is named by the GPJSON_REFERENCE environment variable;
# hosts without it use the prebuilt library that travels with the tree.
REF_KERNELS_REL = Path("gpjson/src/main/resources/com/koenv/gpjson/kernels")


def reference_kernels_dir(reference: str | os.PathLike | None = None) -> Path | None:
    root = reference if reference is not None else os.environ.get("GPJSON_REFERENCE")
    if not root:
        return None
    d = Path(root) / REF_KERNELS_REL
    return d if d.is_dir() else None


def build_reference_kernels(force: bool = False, reference: str | os.PathLike | None = None) -> Path | None:
    """Builds oracle/_ref/libref_gpu.so from the reference's kernel sources
    (`reference`, else $GPJSON_REFERENCE, is the reference checkout) when
    they are present; returns its path, or None without them."""
    target = HERE / "_ref" / "libref_gpu.so"
    kernels = reference_kernels_dir(reference)
    if kernels is None:
        return target if target.exists() else None
    deps = [HERE / "ref_gpu_driver.cu"] + sorted(kernels.glob("*.cu"))
    if force or not target.exists() or any(d.stat().st_mtime > target.stat().st_mtime for d in deps):
        subprocess.run(["make", "-s", "-C", str(HERE), f"REF_KERNELS={kernels}", "_ref/libref_gpu.so"], check=True)
    return target


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = c_void_p
        for name in ("gpjo_newline_index", "gpjo_newline_index_mt"):
            getattr(L, name).restype = c_int64
            getattr(L, name).argtypes = [P, c_int64, P, c_int64]
        for name in ("gpjo_string_index", "gpjo_string_index_mt"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [P, c_int64, P]
        for name in ("gpjo_leveled_bitmaps", "gpjo_leveled_bitmaps_mt"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [P, c_int64, P, c_int, P]
        for name in ("gpjo_find_value", "gpjo_find_value_mt"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [P, c_int64, P, c_int64, P, P, c_int, P, c_int64, c_int, P]
        L.gpjo_num_threads.restype = c_int
        L.gpjo_num_threads.argtypes = []
        _lib = L
    return _lib


def _u8(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data, dtype=np.uint8)
    return np.frombuffer(bytes(data), dtype=np.uint8)


def num_threads() -> int:
    return lib().gpjo_num_threads()


def newline_index(data, mt: bool = False) -> np.ndarray:
    f = _u8(data)
    fn = lib().gpjo_newline_index_mt if mt else lib().gpjo_newline_index
    cnt = fn(f.ctypes.data, f.size, None, 0)
    out = np.empty(cnt, dtype=np.int64)
    fn(f.ctypes.data, f.size, out.ctypes.data, cnt)
    return out


def string_index(data, mt: bool = False) -> np.ndarray:
    f = _u8(data)
    out = np.zeros((f.size + 63) // 64, dtype=np.uint64)
    (lib().gpjo_string_index_mt if mt else lib().gpjo_string_index)(f.ctypes.data, f.size, out.ctypes.data)
    return out


def leveled_bitmaps(data, str_index: np.ndarray, num_levels: int, mt: bool = False) -> np.ndarray:
    f = _u8(data)
    words = (f.size + 63) // 64
    out = np.zeros(words * num_levels, dtype=np.uint64)
    fn = lib().gpjo_leveled_bitmaps_mt if mt else lib().gpjo_leveled_bitmaps
    fn(f.ctypes.data, f.size, str_index.ctypes.data, num_levels, out.ctypes.data)
    return out.reshape(num_levels, words)


def find_value(data, nl, str_index, lvl, num_levels, bytecode: bytes, slots: int, mt: bool = False) -> np.ndarray:
    """One query (Sequential.findValue); returns int64 [lines][slots][2]."""
    f = _u8(data)
    ir = np.frombuffer(bytecode, dtype=np.uint8)
    out = np.empty(len(nl) * 2 * slots, dtype=np.int64)
    lvl = np.ascontiguousarray(lvl)
    fn = lib().gpjo_find_value_mt if mt else lib().gpjo_find_value
    fn(f.ctypes.data, f.size, nl.ctypes.data, len(nl), str_index.ctypes.data, lvl.ctypes.data,
       num_levels, ir.ctypes.data, len(ir), slots, out.ctypes.data)
    return out.reshape(len(nl), slots, 2)


def compile_path(path: str):
    """(bytecode, max_depth, num_results) from the Python compiler restatement."""
    return jsonpath_oracle.compile_path(path)


class Index:
    def __init__(self, data, num_levels: int, mt: bool = False):
        self.data = _u8(data)
        self.num_levels = num_levels
        self.newlines = newline_index(self.data, mt)
        self.strings = string_index(self.data, mt)
        self.levels = leveled_bitmaps(self.data, self.strings, num_levels, mt)


def query(data, paths: list[str], mt: bool = False, index: Index | None = None) -> np.ndarray:
    """QueryFunction semantics with each query evaluated alone:
    int64 [nq][lines][max slots][2]."""
    compiled = [compile_path(p) for p in paths]
    depth = max(c[1] for c in compiled)
    slots = max(c[2] for c in compiled)
    idx = index if index is not None and index.num_levels >= depth else Index(data, depth, mt)
    out = np.empty((len(paths), len(idx.newlines), slots, 2), dtype=np.int64)
    for q, (bc, _, _) in enumerate(compiled):
        out[q] = find_value(idx.data, idx.newlines, idx.strings, idx.levels, idx.num_levels, bc, slots, mt)
    return out
