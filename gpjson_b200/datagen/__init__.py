"""Seeded synthetic NDJSON of the benchmark shapes (ndjson_gen.c).

``tweets(nbytes, seed, p_empty_hashtags)`` — tweet-like lines (~1.6 KB mean,
depth 4); ``adversarial(nbytes, seed)`` — line lengths log-uniform
100 B-1 MiB, nesting 1-16, backslash runs, with the fields a.b.c.d, arr[5]
and x[0].y[2].z present with 10-50% misses.  Seeds default to
0x67706a73 + config id.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

_LIB = Path(__file__).resolve().parent.parent / "_native" / "libgpjson_datagen.so"
_lib = None

SEED_BASE = 0x67706A73


def _load():
    global _lib
    if _lib is None:
        if not _LIB.exists():
            from .. import build

            build.build_datagen()
        L = ctypes.CDLL(str(_LIB))
        L.gpjgen_tweets.restype = ctypes.c_int64
        L.gpjgen_tweets.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double]
        L.gpjgen_adversarial.restype = ctypes.c_int64
        L.gpjgen_adversarial.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64]
        _lib = L
    return _lib


def tweets(nbytes: int, seed: int = SEED_BASE + 0, p_empty_hashtags: float = 0.3, out: np.ndarray | None = None) -> np.ndarray:
    buf = np.empty(nbytes, dtype=np.uint8) if out is None else out
    _load().gpjgen_tweets(buf.ctypes.data, nbytes, seed, p_empty_hashtags)
    return buf


def adversarial(nbytes: int, seed: int = SEED_BASE + 2, out: np.ndarray | None = None) -> np.ndarray:
    buf = np.empty(nbytes, dtype=np.uint8) if out is None else out
    _load().gpjgen_adversarial(buf.ctypes.data, nbytes, seed)
    return buf
