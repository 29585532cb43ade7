"""gpjson_b200 — B200-native structural index and JSONPath queries over NDJSON.

Python mirror of GPJSON's polyglot library object (what
``Polyglot.eval('gpjson', 'jsonpath')`` returns, GPJSONLibrary.java:48-54):

    gpjson = GPJSON()
    result = gpjson.query("dataset.json", "$.user.lang")
    result[0][line][0]  # -> str (UTF-8 slice of the line) or None

``query(file, paths, options)`` follows QueryFunction.call
(functions/QueryFunction.java:48-265): a path or a list of 1..255 paths, an
optional options mapping, and a Result indexed [query][line][slot] whose
items are the matched values as strings or None (result/Result.java,
ResultArray.java, ResultItem.java).  Everything runs on the GPU through the
native library; there is no CPU path.
"""

from __future__ import annotations

import ctypes
import json
import mmap
import os
from collections.abc import Sequence
from ctypes import POINTER, byref, c_char_p, c_int, c_int64, c_size_t, c_uint8, c_void_p

import numpy as np

from . import _lib

__all__ = [
    "GPJSON",
    "GPJSONException",
    "JSONPathException",
    "UnsupportedJSONPathException",
    "CompiledQuery",
    "File",
    "Result",
    "ResultArray",
    "ResultItem",
    "compile_path",
    "prepare_queries",
]

MAX_QUERIES = _lib.GPJ_MAX_QUERIES
MAX_LEVELS = _lib.GPJ_MAX_LEVELS


class GPJSONException(Exception):
    """GPJSONException.java: any failure of a query call.  ``code`` is the
    native status (GPJ_E*)."""

    def __init__(self, message: str, code: int = _lib.GPJ_EINVAL):
        super().__init__(message)
        self.code = code


class JSONPathException(GPJSONException):
    """jsonpath/JSONPathException.java: the path does not parse."""


class UnsupportedJSONPathException(JSONPathException):
    """jsonpath/UnsupportedJSONPathException.java: valid JSONPath outside
    the supported subset ([*], .., [a,b], other filters)."""


class CompiledQuery:
    """JSONPathResult.java: bytecode, max depth and number of result stores."""

    __slots__ = ("path", "bytecode", "max_depth", "num_results")

    def __init__(self, path: str, bytecode: bytes, max_depth: int, num_results: int):
        self.path = path
        self.bytecode = bytecode
        self.max_depth = max_depth
        self.num_results = num_results

    def __repr__(self) -> str:
        return f"CompiledQuery({self.path!r}, depth={self.max_depth}, results={self.num_results})"


# JSONPath beyond the reference's subset (GPJ_PATH_* flags; none by default)
PATH_INDEX_UNIONS = 1


def compile_path(path: str, extensions: int = 0) -> CompiledQuery:
    """JSONPathParser(path).compile() via the native compiler; `extensions`
    (PATH_* flags) admits paths beyond the reference's subset."""
    lib = _lib.load()
    cap = 4096 + 16 * len(path.encode("utf-8"))
    while True:
        out = (c_uint8 * cap)()
        n, depth, res = c_size_t(), c_int(), c_int()
        err = ctypes.create_string_buffer(512)
        rc = lib.gpj_compile_ex(path.encode("utf-8"), extensions, out, cap, byref(n), byref(depth), byref(res), err,
                                512)
        if rc == _lib.GPJ_ELIMIT and n.value > cap:
            cap = n.value
            continue
        break
    msg = err.value.decode("utf-8", "replace")
    if rc == _lib.GPJ_EUNSUPPORTED:
        raise UnsupportedJSONPathException(msg, rc)
    if rc == _lib.GPJ_EPARSE:
        raise JSONPathException(msg, rc)
    if rc != _lib.GPJ_OK:
        raise GPJSONException(msg or f"gpj_compile failed ({rc})", rc)
    return CompiledQuery(path, bytes(out[: n.value]), depth.value, res.value)


class ResultItem(Sequence):
    """result/ResultItem.java:32-52: the slots of one line for one query."""

    __slots__ = ("_array", "_line")

    def __init__(self, array: "ResultArray", line: int):
        self._array = array
        self._line = line

    def __len__(self) -> int:
        return self._array.results_per_line

    def offsets(self, slot: int) -> tuple[int, int]:
        o = self._array.offsets[self._line, slot]
        return int(o[0]), int(o[1])

    def __getitem__(self, slot):
        if isinstance(slot, slice):
            return [self[i] for i in range(*slot.indices(len(self)))]
        if slot < 0:
            slot += len(self)
        if not 0 <= slot < len(self):
            raise IndexError(slot)
        start, end = self.offsets(slot)
        if start == -1:
            return None
        if end < start:
            # The reference builds new byte[end - start] here and fails with
            # NegativeArraySizeException (ResultItem.java:47).
            raise GPJSONException(f"result ({start}, {end}) has no end offset")
        return self._array.file_bytes[start:end].decode("utf-8", "replace")


class ResultArray(Sequence):
    """result/ResultArray.java: one query's results, indexed by line."""

    def __init__(self, offsets: np.ndarray, file_bytes):
        self.offsets = offsets  # [lines][slots][2]
        self.file_bytes = file_bytes
        self.results_per_line = offsets.shape[1]

    def __len__(self) -> int:
        return self.offsets.shape[0]

    def __getitem__(self, line):
        if isinstance(line, slice):
            return [self[i] for i in range(*line.indices(len(self)))]
        if line < 0:
            line += len(self)
        if not 0 <= line < len(self):
            raise IndexError(line)
        return ResultItem(self, line)


class Result(Sequence):
    """result/Result.java: [query] -> ResultArray.  ``offsets`` is the raw
    int64 array [queries][lines][slots][2] (start, end), -1 for a miss."""

    def __init__(self, offsets: np.ndarray, file_bytes, paths: list[str]):
        self.offsets = offsets
        self.file_bytes = file_bytes
        self.paths = paths

    @property
    def number_of_lines(self) -> int:
        return self.offsets.shape[1]

    def __len__(self) -> int:
        return self.offsets.shape[0]

    def __getitem__(self, q):
        if isinstance(q, slice):
            return [self[i] for i in range(*q.indices(len(self)))]
        if q < 0:
            q += len(self)
        if not 0 <= q < len(self):
            raise IndexError(q)
        return ResultArray(self.offsets[q], self.file_bytes)


VALUE_NULL, VALUE_PRESENT, VALUE_UNREADABLE = 0, 1, 2


class Values(Sequence):
    """Values gathered on the device (gpj_query_values): [query][line][slot]
    -> str | None with ResultItem's semantics (result/ResultItem.java:32-52),
    read from one compact buffer instead of the file.  ``kinds`` is uint8
    [queries][lines][slots] (VALUE_*), ``offsets`` int64 [items + 1] into
    ``data``."""

    def __init__(self, kinds: np.ndarray, offsets: np.ndarray, data: bytes, paths: list[str]):
        self.kinds = kinds
        self.offsets = offsets
        self.data = data
        self.paths = paths

    def __len__(self) -> int:
        return self.kinds.shape[0]

    def value(self, q: int, line: int, slot: int):
        kind = int(self.kinds[q, line, slot])
        if kind == VALUE_NULL:
            return None
        if kind == VALUE_UNREADABLE:
            raise GPJSONException(f"result of query {q}, line {line}, slot {slot} has no end offset")
        i = (q * self.kinds.shape[1] + line) * self.kinds.shape[2] + slot
        return self.data[int(self.offsets[i]):int(self.offsets[i + 1])].decode("utf-8", "replace")

    def __getitem__(self, q):
        if isinstance(q, slice):
            return [self[i] for i in range(*q.indices(len(self)))]
        if q < 0:
            q += len(self)
        if not 0 <= q < len(self):
            raise IndexError(q)
        return _ValuesArray(self, q)


class _ValuesArray(Sequence):
    def __init__(self, values: Values, q: int):
        self._v, self._q = values, q

    def __len__(self) -> int:
        return self._v.kinds.shape[1]

    def __getitem__(self, line):
        if isinstance(line, slice):
            return [self[i] for i in range(*line.indices(len(self)))]
        if line < 0:
            line += len(self)
        if not 0 <= line < len(self):
            raise IndexError(line)
        return _ValuesItem(self._v, self._q, line)


class _ValuesItem(Sequence):
    def __init__(self, values: Values, q: int, line: int):
        self._v, self._q, self._line = values, q, line

    def __len__(self) -> int:
        return self._v.kinds.shape[2]

    def __getitem__(self, slot):
        if isinstance(slot, slice):
            return [self[i] for i in range(*slot.indices(len(self)))]
        if slot < 0:
            slot += len(self)
        if not 0 <= slot < len(self):
            raise IndexError(slot)
        return self._v.value(self._q, self._line, slot)


def prepare_queries(queries, options=None, extensions: int = 0) -> tuple[list[str], list[CompiledQuery]]:
    """Argument handling and compilation of QueryFunction.call
    (QueryFunction.java:64-136): a path or a list of 1..255 paths, an
    optional mapping with `disable_fallback`, every path compiled, the depth
    within the 16 levels of LeveledBitmapsIndex.  Raises GPJSONException
    (or its JSONPath subclasses) with the reference's messages."""
    if isinstance(queries, str):
        paths = [queries]
    elif isinstance(queries, (list, tuple)):
        if len(queries) > MAX_QUERIES:
            raise GPJSONException("Maximum size of queries is 255", _lib.GPJ_ELIMIT)
        paths = list(queries)
        if not all(isinstance(p, str) for p in paths):
            raise GPJSONException("expected queries to be a string or string array")
    else:
        raise GPJSONException("expected queries to be a string or string array")
    if not paths:
        raise GPJSONException("expected queries to contain at least one query")
    if options is not None and not hasattr(options, "get"):
        raise GPJSONException("Invalid options")
    disable_fallback = bool((options or {}).get("disable_fallback", False))
    compiled = []
    for i, p in enumerate(paths):
        try:
            compiled.append(compile_path(p, extensions))
        except UnsupportedJSONPathException as e:
            how = "fallback disabled" if disable_fallback else "no CPU fallback in this library"
            raise UnsupportedJSONPathException(f"Unsupported JSON path ({i}, {how}): {e}", e.code) from e
        except JSONPathException as e:
            raise JSONPathException(f"Failed to parse JSON path ({i}): {e}", e.code) from e
    depth = max(q.max_depth for q in compiled)
    if depth > MAX_LEVELS:
        raise GPJSONException(f"Invalid number of levels: {depth}", _lib.GPJ_ELIMIT)
    return paths, compiled


class _Native:
    """A native context (gpj_ctx*)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = c_void_p()
        rc = self.lib.gpj_create(device, byref(h))
        if rc != _lib.GPJ_OK:
            raise GPJSONException(self.lib.gpj_last_error(None).decode("utf-8", "replace"), rc)
        self.h = h

    def check(self, rc: int) -> None:
        if rc != _lib.GPJ_OK:
            msg = self.lib.gpj_last_error(self.h).decode("utf-8", "replace")
            if rc == _lib.GPJ_EUNSUPPORTED:
                raise UnsupportedJSONPathException(msg, rc)
            if rc == _lib.GPJ_EPARSE:
                raise JSONPathException(msg, rc)
            raise GPJSONException(msg, rc)

    def close(self) -> None:
        if self.h:
            self.lib.gpj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class File:
    """An NDJSON input resident in device memory together with its index
    (the reference keeps fileMemory and the index buffers for one call:
    QueryFunction.java:148-245)."""

    def __init__(self, native: _Native, handle: c_void_p, host_bytes=None, keepalive=None):
        self._native = native
        self._h = handle
        self.host_bytes = host_bytes
        self._keepalive = keepalive

    @property
    def size(self) -> int:
        return self._native.lib.gpj_file_size(self._h)

    def build_index(self, num_levels: int) -> None:
        """CombinedIndex.create + LeveledBitmapsIndex(num_levels).create."""
        self._native.check(self._native.lib.gpj_index_build(self._native.h, self._h, num_levels))

    @property
    def num_lines(self) -> int:
        n = c_int64()
        self._native.check(self._native.lib.gpj_index_num_lines(self._h, byref(n)))
        return n.value

    def newline_index(self) -> np.ndarray:
        lines = self.num_lines
        out = np.empty(lines, dtype=np.int64)
        self._native.check(
            self._native.lib.gpj_index_copy_newlines(self._native.h, self._h, out.ctypes.data, lines)
        )
        return out

    def string_index(self) -> np.ndarray:
        words = (self.size + 63) // 64
        out = np.empty(words, dtype=np.uint64)
        self._native.check(
            self._native.lib.gpj_index_copy_string_index(self._native.h, self._h, out.ctypes.data, words)
        )
        return out

    def leveled_bitmaps(self, num_levels: int) -> np.ndarray:
        words = (self.size + 63) // 64
        out = np.empty(words * num_levels, dtype=np.uint64)
        self._native.check(
            self._native.lib.gpj_index_copy_leveled_bitmaps(self._native.h, self._h, out.ctypes.data, out.size)
        )
        return out.reshape(num_levels, words)

    def run(self, queries: list[CompiledQuery], slots: int | None = None) -> np.ndarray:
        """One fused find_value pass; returns int64 [nq][lines][slots][2]."""
        nq = len(queries)
        slots = slots or max(q.num_results for q in queries)
        bufs = [ctypes.create_string_buffer(q.bytecode, len(q.bytecode)) for q in queries]
        ptrs = (c_void_p * nq)(*[ctypes.addressof(b) for b in bufs])
        lens = (c_size_t * nq)(*[len(q.bytecode) for q in queries])
        out = np.empty((nq, self.num_lines, slots, 2), dtype=np.int64)
        self._native.check(
            self._native.lib.gpj_query(self._native.h, self._h, nq, ptrs, lens, slots, out.ctypes.data, out.size)
        )
        return out

    def query_paths(self, paths: list[str]) -> np.ndarray:
        """gpj_query_paths: compile, index and evaluate in one pass (an index
        already built with enough levels is reused); returns int64
        [nq][lines][slots][2]."""
        arr = (c_char_p * len(paths))(*[p.encode("utf-8") for p in paths])
        r = c_void_p()
        self._native.check(self._native.lib.gpj_query_paths(self._native.h, self._h, len(paths), arr, byref(r)))
        return _result_array(self._native.lib, r)

    def query_values(self, paths: list[str]) -> Values:
        """gpj_query_values: the paths evaluated as by query_paths and the
        matched values gathered on the device (no host read of the file)."""
        arr = (c_char_p * len(paths))(*[p.encode("utf-8") for p in paths])
        v = c_void_p()
        self._native.check(self._native.lib.gpj_query_values(self._native.h, self._h, len(paths), arr, byref(v)))
        lib = self._native.lib
        # kinds and offsets stay in the native object (numpy views own it);
        # the value bytes are copied once, into the bytes object Values holds
        owner = _NativeOwner(lib.gpj_values_release, v)
        nq, lines, slots = lib.gpj_values_num_queries(v), lib.gpj_values_num_lines(v), lib.gpj_values_slots(v)
        items = nq * lines * slots
        kinds = _native_view(owner, lib.gpj_values_kinds(v), items, "|u1")
        offsets = _native_view(owner, lib.gpj_values_offsets(v), items + 1, "<i8")
        size = lib.gpj_values_size(v)
        data = ctypes.string_at(lib.gpj_values_bytes(v), size) if size else b""
        return Values(kinds.reshape(nq, lines, slots), offsets, data, list(paths))

    def index_and_query_device(self, queries: list[CompiledQuery], num_levels: int, d_out: int, out_lines: int,
                               slots: int | None = None) -> None:
        """gpj_index_query_device: index + queries in one pass into device
        memory at address d_out (int64 [nq][out_lines][slots][2])."""
        nq = len(queries)
        slots = slots or max(q.num_results for q in queries)
        bufs = [ctypes.create_string_buffer(q.bytecode, len(q.bytecode)) for q in queries]
        ptrs = (c_void_p * nq)(*[ctypes.addressof(b) for b in bufs])
        lens = (c_size_t * nq)(*[len(q.bytecode) for q in queries])
        self._native.check(self._native.lib.gpj_index_query_device(
            self._native.h, self._h, num_levels, nq, ptrs, lens, slots, c_void_p(d_out), out_lines))

    def release(self) -> None:
        if self._h:
            self._native.lib.gpj_file_release(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class _NativeOwner:
    """Owns a native object (gpj_result, gpj_values) and releases it when
    the last numpy view of its memory is collected."""

    def __init__(self, release, handle):
        self._release, self._h = release, handle

    def __del__(self):
        if self._h:
            self._release(self._h)
            self._h = None


class _NativeView:
    """`count` elements of numpy type `typestr` at `addr`, memory owned by
    `owner`; np.asarray of it is a view that keeps the owner alive."""

    def __init__(self, owner: _NativeOwner, addr: int, count: int, typestr: str):
        self._owner = owner
        self.__array_interface__ = {"shape": (count,), "typestr": typestr, "data": (addr, False), "version": 3}


def _native_view(owner: _NativeOwner, addr, count: int, typestr: str) -> np.ndarray:
    if count == 0:
        return np.zeros(0, dtype=np.dtype(typestr))
    return np.asarray(_NativeView(owner, addr, count, typestr))


def _result_array(lib, r) -> np.ndarray:
    """int64 [nq][lines][slots][2] over a gpj_result's offsets (no copy: the
    array owns the result and releases it when it is collected)."""
    owner = _NativeOwner(lib.gpj_result_release, r)
    nq, lines, slots = lib.gpj_result_num_queries(r), lib.gpj_result_num_lines(r), lib.gpj_result_slots(r)
    count = nq * lines * slots * 2
    return _native_view(owner, lib.gpj_result_offsets(r), count, "<i8").reshape(nq, lines, slots, 2)


class Batch:
    """gpj_batch: many (file, paths) requests indexed and evaluated together
    (one index launch for the files that need it, one find_value launch, one
    copy back).  Each request's results equal File.query_paths on its file."""

    def __init__(self, native: "_Native"):
        self._native = native
        self._h = c_void_p()
        native.check(native.lib.gpj_batch_create(native.h, byref(self._h)))
        self._files: list[File] = []  # kept alive until the batch is cleared

    def add(self, file: "File", paths: list[str]) -> int:
        arr = (c_char_p * len(paths))(*[p.encode("utf-8") for p in paths])
        item = c_int()
        self._native.check(self._native.lib.gpj_batch_add(self._h, file._h, len(paths), arr, byref(item)))
        self._files.append(file)
        return item.value

    def run(self) -> None:
        self._native.check(self._native.lib.gpj_batch_run(self._h))

    def result(self, item: int) -> np.ndarray:
        """int64 [nq][lines][slots][2] of request `item`."""
        r = c_void_p()
        self._native.check(self._native.lib.gpj_batch_result(self._h, item, byref(r)))
        return _result_array(self._native.lib, r)

    def __len__(self) -> int:
        return self._native.lib.gpj_batch_size(self._h)

    def clear(self) -> None:
        self._native.lib.gpj_batch_clear(self._h)
        self._files.clear()

    def release(self) -> None:
        if self._h:
            self._native.lib.gpj_batch_release(self._h)
            self._h = c_void_p()
            self._files.clear()


class GPJSON:
    """The library object of GPJSONLibrary.java: members ``query`` and
    ``exportTimings``."""

    def __init__(self, device: int = 0):
        self._native = _Native(device)
        self._extensions = 0

    # -- files ---------------------------------------------------------------
    def open(self, filename: str | os.PathLike) -> File:
        h = c_void_p()
        self._native.check(self._native.lib.gpj_file_open(self._native.h, os.fsencode(filename), byref(h)))
        return File(self._native, h)

    def load_bytes(self, data: bytes | bytearray | memoryview | np.ndarray) -> File:
        arr = np.frombuffer(data, dtype=np.uint8) if not isinstance(data, np.ndarray) else data
        h = c_void_p()
        self._native.check(
            self._native.lib.gpj_file_from_host(self._native.h, arr.ctypes.data, arr.size, byref(h))
        )
        return File(self._native, h, host_bytes=bytes(arr.tobytes()) if arr.size < (1 << 26) else arr)

    def load_bytes_indexed(self, data: bytes | bytearray | memoryview | np.ndarray, num_levels: int) -> File:
        """gpj_file_from_host_indexed: copy and index in one pipelined call."""
        arr = np.frombuffer(data, dtype=np.uint8) if not isinstance(data, np.ndarray) else data
        h = c_void_p()
        self._native.check(self._native.lib.gpj_file_from_host_indexed(
            self._native.h, arr.ctypes.data, arr.size, num_levels, byref(h)))
        return File(self._native, h, host_bytes=bytes(arr.tobytes()) if arr.size < (1 << 26) else arr)

    def load_bytes_query(self, data: bytes | bytearray | memoryview | np.ndarray, num_levels: int,
                         queries: list[CompiledQuery], slots: int | None = None,
                         out: np.ndarray | None = None) -> tuple[File, np.ndarray]:
        """gpj_file_from_host_query: copy, index and query in one pipelined
        call; returns the indexed File and int64 [nq][lines][slots][2].
        `out` (optional, e.g. page-locked) receives the results when it is
        large enough; otherwise a new array is returned."""
        arr = np.frombuffer(data, dtype=np.uint8) if not isinstance(data, np.ndarray) else data
        nq = len(queries)
        slots = slots or max(q.num_results for q in queries)
        bufs = [ctypes.create_string_buffer(q.bytecode, len(q.bytecode)) for q in queries]
        ptrs = (c_void_p * nq)(*[ctypes.addressof(b) for b in bufs])
        lens = (c_size_t * nq)(*[len(q.bytecode) for q in queries])
        h, lines = c_void_p(), c_int64()
        dst = out if out is not None else np.empty(0, dtype=np.int64)
        rc = self._native.lib.gpj_file_from_host_query(
            self._native.h, arr.ctypes.data, arr.size, num_levels, nq, ptrs, lens, slots,
            dst.ctypes.data if dst.size else None, dst.size, byref(lines), byref(h))
        if rc == _lib.GPJ_ELIMIT and h.value:
            f = File(self._native, h, host_bytes=bytes(arr.tobytes()) if arr.size < (1 << 26) else arr)
            return f, f.run(queries, slots)
        self._native.check(rc)
        f = File(self._native, h, host_bytes=bytes(arr.tobytes()) if arr.size < (1 << 26) else arr)
        return f, dst.reshape(-1)[: nq * lines.value * slots * 2].reshape(nq, lines.value, slots, 2)

    def from_device(self, ptr: int, n: int, keepalive=None) -> File:
        """Wraps n bytes already in device memory (e.g. a torch uint8 tensor's
        data_ptr()); `keepalive` is held for the File's lifetime."""
        h = c_void_p()
        self._native.check(self._native.lib.gpj_file_from_device(self._native.h, c_void_p(ptr), n, byref(h)))
        return File(self._native, h, keepalive=keepalive)

    def batch(self) -> Batch:
        return Batch(self._native)

    def set_path_extensions(self, extensions: int) -> None:
        """JSONPath extensions (PATH_* flags) for the calls that take path
        strings (query, query_paths, query_values, batches); 0 = the
        reference's subset exactly."""
        self._native.check(self._native.lib.gpj_set_path_extensions(self._native.h, extensions))
        self._extensions = extensions

    def set_query_fusion(self, enabled: bool) -> None:
        """Evaluate queries inside the index kernel (True) or with one
        find_value launch after it (False, the default)."""
        self._native.check(self._native.lib.gpj_set_query_fusion(self._native.h, 1 if enabled else 0))

    def tuning(self) -> dict:
        """gpj_get_tuning: the context's launch shapes."""
        t = _lib.Tuning()
        self._native.check(self._native.lib.gpj_get_tuning(self._native.h, byref(t)))
        return {"long_line_bytes": t.long_line_bytes, "query_ctas_per_sm": t.query_ctas_per_sm,
                "index_ctas_per_sm": t.index_ctas_per_sm, "chunk_tiles": t.chunk_tiles}

    def set_tuning(self, long_line_bytes: int | None = None, query_ctas_per_sm: int | None = None,
                   index_ctas_per_sm: int | None = None, chunk_tiles: int | None = None) -> None:
        """gpj_set_tuning: changes the given launch shapes (results do not
        depend on them)."""
        cur = self.tuning()
        t = _lib.Tuning(cur["long_line_bytes"] if long_line_bytes is None else long_line_bytes,
                        cur["query_ctas_per_sm"] if query_ctas_per_sm is None else query_ctas_per_sm,
                        cur["index_ctas_per_sm"] if index_ctas_per_sm is None else index_ctas_per_sm,
                        cur["chunk_tiles"] if chunk_tiles is None else chunk_tiles, 0)
        self._native.check(self._native.lib.gpj_set_tuning(self._native.h, byref(t)))

    def set_stream(self, stream_handle: int | None) -> None:
        self._native.check(self._native.lib.gpj_set_stream(self._native.h, c_void_p(stream_handle or 0)))

    # -- the reference members ------------------------------------------------
    def query(self, filename, queries, options=None) -> Result:
        """QueryFunction.call: query(file, path | [paths], options?)."""
        paths, _ = prepare_queries(queries, options, self._extensions)
        f = self.open(filename)
        try:
            offsets = f.query_paths(paths)
        finally:
            f.release()
        with open(filename, "rb") as fh:
            size = os.fstat(fh.fileno()).st_size
            file_bytes = mmap.mmap(fh.fileno(), 0, access=mmap.ACCESS_READ) if size else b""
        return Result(offsets, file_bytes, paths)

    def query_values(self, filename, queries, options=None) -> Values:
        """query() with the matched values gathered on the device
        (gpj_query_values): the same [query][line][slot] -> str | None view,
        without reading the file again on the host."""
        paths, _ = prepare_queries(queries, options, self._extensions)
        f = self.open(filename)
        try:
            return f.query_values(paths)
        finally:
            f.release()

    def exportTimings(self) -> str:  # noqa: N802  (reference member name)
        """ExportTimingsFunction: the context's phase timings as JSON."""
        n = c_size_t()
        self._native.lib.gpj_get_timings(self._native.h, None, 0, byref(n))
        buf = ctypes.create_string_buffer(n.value + 1)
        self._native.check(self._native.lib.gpj_get_timings(self._native.h, buf, n.value + 1, byref(n)))
        return buf.value.decode()

    def timings(self) -> dict:
        return json.loads(self.exportTimings())

    def kernel_launches(self) -> int:
        return self._native.lib.gpj_kernel_launches(self._native.h)

    def close(self) -> None:
        self._native.close()
