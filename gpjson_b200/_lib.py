"""ctypes binding of the C ABI declared in include/gpjson_b200.h.

This is the Python counterpart of the binding a Java caller makes with the
Panama FFM API.  Loading fails loudly when the native library has not been
built: there is no CPU implementation behind this package.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_int, c_int64, c_size_t, c_uint, c_uint8, c_uint64, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_native" / "libgpjson_b200.so"
# A different build of the same library (e.g. for profiling experiments).
_LIB_OVERRIDE = "GPJSON_B200_LIB"

GPJ_OK = 0
GPJ_EINVAL = -1
GPJ_EPARSE = -2
GPJ_EUNSUPPORTED = -3
GPJ_ECUDA = -4
GPJ_ENOMEM = -5
GPJ_EIO = -6
GPJ_ELIMIT = -7
GPJ_EDEVICE = -8
GPJ_ESTATE = -9
GPJ_EAGAIN = -10

GPJ_MAX_QUERIES = 255
GPJ_MAX_LEVELS = 16

class Tuning(ctypes.Structure):
    """gpj_tuning: launch shapes of a context's kernels."""

    _fields_ = [("long_line_bytes", c_int64), ("query_ctas_per_sm", ctypes.c_int32),
                ("index_ctas_per_sm", ctypes.c_int32), ("chunk_tiles", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class ServerConfig(ctypes.Structure):
    """gpj_server_config."""

    _fields_ = [("device", ctypes.c_int32), ("num_levels", ctypes.c_int32), ("budget_bytes", c_int64),
                ("max_batch", ctypes.c_int32), ("workers", ctypes.c_int32)]


# name -> (restype, argtypes); the full list of exported entry points.
SIGNATURES: dict[str, tuple] = {
    "gpj_create": (c_int, [c_int, POINTER(c_void_p)]),
    "gpj_destroy": (None, [c_void_p]),
    "gpj_last_error": (c_char_p, [c_void_p]),
    "gpj_set_stream": (c_int, [c_void_p, c_void_p]),
    "gpj_version": (c_char_p, []),
    "gpj_compile": (
        c_int,
        [c_char_p, POINTER(c_uint8), c_size_t, POINTER(c_size_t), POINTER(c_int), POINTER(c_int), c_char_p, c_size_t],
    ),
    "gpj_file_open": (c_int, [c_void_p, c_char_p, POINTER(c_void_p)]),
    "gpj_file_from_host": (c_int, [c_void_p, c_void_p, c_int64, POINTER(c_void_p)]),
    "gpj_file_from_device": (c_int, [c_void_p, c_void_p, c_int64, POINTER(c_void_p)]),
    "gpj_file_release": (None, [c_void_p]),
    "gpj_file_size": (c_int64, [c_void_p]),
    "gpj_index_build": (c_int, [c_void_p, c_void_p, c_int]),
    "gpj_index_num_lines": (c_int, [c_void_p, POINTER(c_int64)]),
    "gpj_index_copy_newlines": (c_int, [c_void_p, c_void_p, c_void_p, c_int64]),
    "gpj_index_copy_string_index": (c_int, [c_void_p, c_void_p, c_void_p, c_int64]),
    "gpj_index_copy_leveled_bitmaps": (c_int, [c_void_p, c_void_p, c_void_p, c_int64]),
    "gpj_build_index_device": (
        c_int,
        [c_void_p, c_void_p, c_int64, c_int, c_void_p, c_void_p, c_void_p, c_int64, POINTER(c_int64)],
    ),
    "gpj_build_index_device_noalloc": (
        c_int,
        [c_void_p, c_void_p, c_int64, c_int, c_void_p, c_void_p, c_void_p, c_int64, POINTER(c_int64)],
    ),
    "gpj_set_query_fusion": (c_int, [c_void_p, c_int]),
    "gpj_set_tuning": (c_int, [c_void_p, POINTER(Tuning)]),
    "gpj_get_tuning": (c_int, [c_void_p, POINTER(Tuning)]),
    "gpj_set_path_extensions": (c_int, [c_void_p, c_uint]),
    "gpj_compile_ex": (
        c_int,
        [c_char_p, c_uint, POINTER(c_uint8), c_size_t, POINTER(c_size_t), POINTER(c_int), POINTER(c_int),
         c_char_p, c_size_t],
    ),
    "gpj_file_from_host_indexed": (c_int, [c_void_p, c_void_p, c_int64, c_int, POINTER(c_void_p)]),
    "gpj_file_from_host_query": (
        c_int,
        [c_void_p, c_void_p, c_int64, c_int, c_int, POINTER(c_void_p), POINTER(c_size_t), c_int, c_void_p, c_int64,
         POINTER(c_int64), POINTER(c_void_p)],
    ),
    "gpj_batch_create": (c_int, [c_void_p, POINTER(c_void_p)]),
    "gpj_batch_add": (c_int, [c_void_p, c_void_p, c_int, POINTER(c_char_p), POINTER(c_int)]),
    "gpj_batch_run": (c_int, [c_void_p]),
    "gpj_batch_result": (c_int, [c_void_p, c_int, POINTER(c_void_p)]),
    "gpj_batch_result_ex": (c_int, [c_void_p, c_int, c_int, POINTER(c_void_p)]),
    "gpj_serve_create": (c_int, [POINTER(ServerConfig), POINTER(c_void_p)]),
    "gpj_serve_add_corpus": (c_int, [c_void_p, c_void_p, c_int64, POINTER(c_int)]),
    "gpj_serve_set_batching": (c_int, [c_void_p, c_int, c_int]),
    "gpj_serve_submit": (c_int, [c_void_p, c_int, c_int, POINTER(c_char_p), POINTER(c_uint64)]),
    "gpj_serve_poll": (
        c_int, [c_void_p, c_uint64, c_int, POINTER(c_void_p), POINTER(c_int64), POINTER(c_int64)]
    ),
    "gpj_serve_now_ns": (c_int64, [c_void_p]),
    "gpj_serve_stats": (c_int, [c_void_p, c_char_p, c_size_t, POINTER(c_size_t)]),
    "gpj_serve_destroy": (None, [c_void_p]),
    "gpj_batch_size": (c_int, [c_void_p]),
    "gpj_batch_clear": (None, [c_void_p]),
    "gpj_batch_release": (None, [c_void_p]),
    "gpj_query": (c_int, [c_void_p, c_void_p, c_int, POINTER(c_void_p), POINTER(c_size_t), c_int, c_void_p, c_int64]),
    "gpj_query_device": (
        c_int,
        [c_void_p, c_void_p, c_int, POINTER(c_void_p), POINTER(c_size_t), c_int, c_void_p, c_int64],
    ),
    "gpj_index_query_device": (
        c_int,
        [c_void_p, c_void_p, c_int, c_int, POINTER(c_void_p), POINTER(c_size_t), c_int, c_void_p, c_int64],
    ),
    "gpj_query_paths": (c_int, [c_void_p, c_void_p, c_int, POINTER(c_char_p), POINTER(c_void_p)]),
    "gpj_result_num_queries": (c_int64, [c_void_p]),
    "gpj_result_num_lines": (c_int64, [c_void_p]),
    "gpj_result_slots": (c_int, [c_void_p]),
    "gpj_result_offsets": (c_void_p, [c_void_p]),
    "gpj_result_release": (None, [c_void_p]),
    "gpj_values_device": (
        c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_int64, POINTER(c_int64)]
    ),
    "gpj_query_values": (c_int, [c_void_p, c_void_p, c_int, POINTER(c_char_p), POINTER(c_void_p)]),
    "gpj_values_num_queries": (c_int64, [c_void_p]),
    "gpj_values_num_lines": (c_int64, [c_void_p]),
    "gpj_values_slots": (c_int, [c_void_p]),
    "gpj_values_kinds": (c_void_p, [c_void_p]),
    "gpj_values_offsets": (c_void_p, [c_void_p]),
    "gpj_values_bytes": (c_void_p, [c_void_p]),
    "gpj_values_size": (c_int64, [c_void_p]),
    "gpj_values_release": (None, [c_void_p]),
    "gpj_get_timings": (c_int, [c_void_p, c_char_p, c_size_t, POINTER(c_size_t)]),
    "gpj_reset_timings": (None, [c_void_p]),
    "gpj_kernel_launches": (c_int64, [c_void_p]),
}

_lib = None


def load(path: str | Path | None = None) -> ctypes.CDLL:
    """Loads (once) and returns the native library with typed signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    import os

    p = Path(path) if path else Path(os.environ.get(_LIB_OVERRIDE, LIB_PATH))
    if not p.exists():
        raise RuntimeError(
            f"gpjson_b200 native library not found at {p}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (needs nvcc)"
        )
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
