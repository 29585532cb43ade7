"""TEST AND MEASUREMENT INFRASTRUCTURE ONLY: ctypes front end of
oracle/_ref/libref_gpu.so, the reference's own CUDA kernels compiled from
source with the reference's orchestration replayed (ref_gpu_driver.cu).
Used by the GPU tests (a second oracle on the device) and by bench.py (the
reference's GPU path timed on the same GPU); never by the gpjson_b200
package.  The library is built where the reference sources are
(oracle/Makefile target _ref/libref_gpu.so) and travels with the tree.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_int64, c_size_t, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libref_gpu.so"
_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        L = ctypes.CDLL(str(LIB_PATH))
        L.ref_gpu_run.restype = c_int
        L.ref_gpu_run.argtypes = [c_void_p, c_int64, c_int, c_int, POINTER(c_void_p), POINTER(c_size_t), c_int, c_int,
                                  c_void_p, c_void_p, c_void_p, c_int64, POINTER(c_int64), c_void_p, c_int64,
                                  POINTER(c_double), POINTER(c_double)]
        _lib = L
    return _lib


def run(data: bytes | np.ndarray, num_levels: int, bytecodes: list[bytes], slots: int, repeats: int = 1,
        outputs: bool = True, max_lines: int | None = None) -> dict:
    """Index + queries with the reference kernels on the GPU.  Returns the
    mean index and query wall times (ms) and, with `outputs`, the string
    index, leveled bitmaps, newline index and results [nq][lines][slots][2]."""
    arr = np.frombuffer(data, dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    n = arr.size
    words = (n + 63) // 64
    nq = len(bytecodes)
    bufs = [ctypes.create_string_buffer(b, len(b)) for b in bytecodes]
    ptrs = (c_void_p * nq)(*[ctypes.addressof(b) for b in bufs])
    lens = (c_size_t * nq)(*[len(b) for b in bytecodes])
    cap = max_lines if max_lines is not None else n + 1
    out = {}
    if outputs:
        out["strings"] = np.zeros(words, dtype=np.uint64)
        out["levels"] = np.zeros(words * num_levels, dtype=np.uint64)
        newlines = np.zeros(cap, dtype=np.int64)
        results = np.zeros(nq * cap * slots * 2, dtype=np.int64)
    lines, t_index, t_query = c_int64(), c_double(), c_double()
    rc = lib().ref_gpu_run(
        arr.ctypes.data, n, num_levels, nq, ptrs, lens, slots, repeats,
        out["strings"].ctypes.data if outputs else None, out["levels"].ctypes.data if outputs else None,
        newlines.ctypes.data if outputs else None, cap, ctypes.byref(lines),
        results.ctypes.data if outputs else None, results.size if outputs else 0,
        ctypes.byref(t_index), ctypes.byref(t_query))
    if rc != 0:
        raise RuntimeError(f"ref_gpu_run failed: {rc}")
    out["index_ms"], out["query_ms"], out["lines"] = t_index.value, t_query.value, lines.value
    if outputs:
        out["levels"] = out["levels"].reshape(num_levels, words)
        out["newlines"] = newlines[: lines.value]
        out["results"] = results[: nq * lines.value * slots * 2].reshape(nq, lines.value, slots, 2)
    return out
