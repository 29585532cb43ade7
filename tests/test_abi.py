"""The C ABI library loads, exports every entry point include/gpjson_b200.h
declares, binds them all in Python, and behaves without a GPU (compiler
calls work; context creation fails with a status, never a crash)."""

from __future__ import annotations

import re
import subprocess

import pytest

import gpjson_b200 as gj
from gpjson_b200 import _lib
from tests.conftest import ROOT

HEADER = ROOT / "include" / "gpjson_b200.h"


def declared_functions() -> set[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return set(re.findall(r"\b(gpj_[a-z_0-9]+)\s*\(", text))


def exported_symbols() -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], check=True, capture_output=True,
                         text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_symbol():
    declared = declared_functions()
    assert len(declared) >= 25
    exported = exported_symbols()
    assert declared <= exported, declared - exported
    # nothing but the declared API leaks out of the library
    assert {s for s in exported if s.startswith("gpj")} == declared


def test_python_binding_covers_header():
    assert set(_lib.SIGNATURES) == declared_functions()
    lib = _lib.load()
    for name in _lib.SIGNATURES:
        assert getattr(lib, name) is not None


def test_version_and_compile_without_gpu():
    lib = _lib.load()
    assert b"sm_100a" in lib.gpj_version()
    c = gj.compile_path("$.user.lang")
    assert c.bytecode[0] == 4 and c.max_depth == 2


def test_null_arguments_are_rejected():
    lib = _lib.load()
    assert lib.gpj_create(0, None) == _lib.GPJ_EINVAL
    assert lib.gpj_index_num_lines(None, None) == _lib.GPJ_EINVAL
    assert lib.gpj_get_timings(None, None, 0, None) == _lib.GPJ_EINVAL
    assert lib.gpj_kernel_launches(None) == -1
    lib.gpj_file_release(None)
    lib.gpj_result_release(None)
    lib.gpj_destroy(None)


def test_context_creation_reports_status():
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present; covered by the gpu tests")
    with pytest.raises(gj.GPJSONException) as ei:
        gj.GPJSON(0)
    assert ei.value.code in (_lib.GPJ_ECUDA, _lib.GPJ_ENOMEM)
    assert "CUDA error" in str(ei.value) or "sm_100" in str(ei.value)


def test_query_argument_handling():
    with pytest.raises(gj.GPJSONException, match="255"):
        gj.prepare_queries(["$.a"] * 256)
    with pytest.raises(gj.GPJSONException, match="at least one"):
        gj.prepare_queries([])
    with pytest.raises(gj.GPJSONException, match="string or string array"):
        gj.prepare_queries(3)
    with pytest.raises(gj.GPJSONException, match="string or string array"):
        gj.prepare_queries(["$.a", 3])
    with pytest.raises(gj.UnsupportedJSONPathException, match=r"Unsupported JSON path \(1, fallback disabled\)"):
        gj.prepare_queries(["$.a", "$[*]"], {"disable_fallback": True})
    with pytest.raises(gj.JSONPathException, match=r"Failed to parse JSON path \(0\)"):
        gj.prepare_queries(["$.a b"])
    with pytest.raises(gj.GPJSONException, match="levels"):
        gj.prepare_queries("$" + ".a" * 17)
    paths, compiled = gj.prepare_queries(("$.a", "$.b[0:2]"))
    assert paths == ["$.a", "$.b[0:2]"] and [c.num_results for c in compiled] == [1, 2]


def test_result_views_follow_reference_layout():
    import numpy as np

    data = b'{"a":"x"}\n{"a":12}\n{"b":1}'
    offs = np.array([[[[5, 8]], [[15, 17]], [[-1, -1]]]], dtype=np.int64)
    r = gj.Result(offs, data, ["$.a"])
    assert len(r) == 1 and len(r[0]) == 3 and len(r[0][0]) == 1
    assert [r[0][i][0] for i in range(3)] == ['"x"', "12", None]
    assert r[-1][-1][-1] is None
    with pytest.raises(IndexError):
        r[1]
    with pytest.raises(IndexError):
        r[0][3]


def test_values_view_follows_result_item():
    """The compact value view (gj.Values) answers like ResultItem: null for
    a miss, the value's text, an error for a pair without an end, UTF-8
    decoded with replacement."""
    import numpy as np

    kinds = np.array([[[gj.VALUE_PRESENT], [gj.VALUE_NULL], [gj.VALUE_UNREADABLE], [gj.VALUE_PRESENT]]],
                     dtype=np.uint8)
    data = '"x"12"été"'.encode() + b"\xff"
    offsets = np.array([0, 3, 3, 3, len(data)], dtype=np.int64)
    v = gj.Values(kinds, offsets, data, ["$.a"])
    assert len(v) == 1 and len(v[0]) == 4 and len(v[0][0]) == 1
    assert v[0][0][0] == '"x"' and v[0][1][0] is None
    with pytest.raises(gj.GPJSONException):
        v[0][2][0]
    assert v[0][3][0] == '12"été"�'
    assert v[-1][-1][:] == ['12"été"�']
    with pytest.raises(IndexError):
        v[0][4]


def test_result_array_is_a_view_that_owns_the_result():
    """Result offsets reach numpy without a copy: the array reads the native
    result's memory, and the result is released once, when the last array
    over it is collected."""
    import ctypes
    import gc

    import numpy as np

    from gpjson_b200 import _result_array

    store = (ctypes.c_int64 * 12)(*range(12))
    released = []

    class FakeLib:  # the gpj_result accessors of the C ABI
        def gpj_result_num_queries(self, r):
            return 2

        def gpj_result_num_lines(self, r):
            return 3

        def gpj_result_slots(self, r):
            return 1

        def gpj_result_offsets(self, r):
            return ctypes.addressof(store)

        def gpj_result_release(self, r):
            released.append(r.value)

    a = _result_array(FakeLib(), ctypes.c_void_p(0x1234))
    assert a.shape == (2, 3, 1, 2) and a.dtype == np.int64
    assert a.reshape(-1).tolist() == list(range(12))
    store[5] = 99  # the array reads the result's memory
    assert a[0, 2, 0, 1] == 99
    q0 = a[0]
    del a
    gc.collect()
    assert released == []  # a slice still holds the result
    assert q0[1, 0, 0] == 2
    del q0
    gc.collect()
    assert released == [0x1234]


@pytest.mark.parametrize("lang,std", [("c", "c99"), ("c++", "c++17")])
def test_header_compiles_standalone(lang, std):
    """include/gpjson_b200.h is a plain C header: a C99 or C++17 caller
    includes it alone, without warnings."""
    cc = "gcc" if lang == "c" else "g++"
    subprocess.run([cc, f"-std={std}", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only", "-x", lang,
                    str(ROOT / "include" / "gpjson_b200.h")], check=True)


def test_host_io_header_compiles_cleanly():
    """The C ABI's host I/O header (parallel file reader, result buffers)
    builds without warnings on its own."""
    header = ROOT / "gpjson_b200" / "csrc" / "host_io.h"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-x", "c++", "-"],
                   input=f'#include "{header}"\n'.encode(), check=True)


def test_values_arrays_are_views_that_own_the_native_values():
    """File.query_values hands the native kinds and offsets to numpy in
    place (the value bytes are copied once into bytes); the gpj_values is
    released once, when the Values and every array taken from it are gone."""
    import ctypes
    import gc

    import numpy as np

    kinds = (ctypes.c_uint8 * 6)(gj.VALUE_PRESENT, gj.VALUE_NULL, gj.VALUE_PRESENT, gj.VALUE_UNREADABLE,
                                 gj.VALUE_PRESENT, gj.VALUE_NULL)
    offs = (ctypes.c_int64 * 7)(0, 3, 3, 5, 5, 10, 10)
    data = ctypes.create_string_buffer(b'"x"12"abc"', 10)
    released = []

    class FakeLib:  # the gpj_query_values / gpj_values_* entry points
        def gpj_query_values(self, ctx, file, nq, paths, out):
            out._obj.value = 0x77
            return 0

        def gpj_values_num_queries(self, v):
            return 2

        def gpj_values_num_lines(self, v):
            return 3

        def gpj_values_slots(self, v):
            return 1

        def gpj_values_kinds(self, v):
            return ctypes.addressof(kinds)

        def gpj_values_offsets(self, v):
            return ctypes.addressof(offs)

        def gpj_values_size(self, v):
            return 10

        def gpj_values_bytes(self, v):
            return ctypes.addressof(data)

        def gpj_values_release(self, v):
            released.append(v.value)

    class FakeNative:
        lib, h = FakeLib(), None

        def check(self, rc):
            assert rc == 0

    f = gj.File(FakeNative(), ctypes.c_void_p(1))
    try:
        vals = f.query_values(["$.a", "$.b"])
    finally:
        f._h = None  # no native file behind the fake
    assert vals.kinds.shape == (2, 3, 1) and vals.data == b'"x"12"abc"'
    assert [vals[0][i][0] for i in range(3)] == ['"x"', None, "12"]
    with pytest.raises(gj.GPJSONException):
        vals[1][0][0]
    assert vals[1][1][0] == '"abc"' and vals[1][2][0] is None
    offs[2] = 2  # the offsets are the native object's memory
    assert vals.offsets[2] == 2
    kept = vals.kinds
    del vals
    gc.collect()
    assert released == []
    assert np.array_equal(kept.reshape(-1), list(kinds))
    del kept
    gc.collect()
    assert released == [0x77]


def test_server_rejects_bad_configuration_without_gpu():
    """gpj_serve_create checks its configuration before any device work."""
    from ctypes import byref, c_void_p

    lib = _lib.load()
    h = c_void_p()
    for cfg in [(0, 0, 1 << 20, 1, 1), (0, 17, 1 << 20, 1, 1), (0, 4, 0, 1, 1), (0, 4, 1 << 20, 0, 1),
                (0, 4, 1 << 20, 1, 0), (0, 4, 1 << 20, 1, 9)]:
        assert lib.gpj_serve_create(byref(_lib.ServerConfig(*cfg)), byref(h)) == _lib.GPJ_EINVAL, cfg
    assert lib.gpj_serve_create(None, byref(h)) == _lib.GPJ_EINVAL
    assert lib.gpj_serve_poll(None, 1, 0, byref(c_void_p()), None, None) == _lib.GPJ_EINVAL
    assert lib.gpj_serve_now_ns(None) == -1
    lib.gpj_serve_destroy(None)
