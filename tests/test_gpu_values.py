"""Device-side value extraction (gpj_query_values, gpj_values_device)
against ResultItem's semantics as the host Result applies them: every item
None, the same string, or unreadable (raises) in both."""

from __future__ import annotations

import numpy as np
import pytest

import gpjson_b200 as gj
from gpjson_b200 import datagen
from tests.conftest import FIXTURES
from tests.test_gpu_query import ADV_PATHS, TWEET_PATHS
from tests.test_oracle import KNOWN_ANSWERS, SIMPLE


def read(item, slot):
    try:
        return ("value", item[slot])
    except gj.GPJSONException:
        return ("unreadable", None)


def assert_same(values: gj.Values, result: gj.Result):
    assert len(values) == len(result)
    for q in range(len(result)):
        va, ra = values[q], result[q]
        assert len(va) == len(ra)
        for line in range(len(ra)):
            vi, ri = va[line], ra[line]
            assert len(vi) == len(ri)
            for slot in range(len(ri)):
                assert read(vi, slot) == read(ri, slot), (q, line, slot)


def values_and_result(gpjson, data: bytes, paths: list[str]):
    f = gpjson.load_bytes(data)
    try:
        values = f.query_values(paths)
        offsets = f.query_paths(paths)
    finally:
        f.release()
    return values, gj.Result(offsets, data, paths)


@pytest.mark.gpu
def test_values_fixture_known_answers(gpjson):
    paths = [k[0] for k in KNOWN_ANSWERS]
    values = gpjson.query_values(str(FIXTURES / SIMPLE), paths)
    result = gpjson.query(str(FIXTURES / SIMPLE), paths)
    assert_same(values, result)
    for q, (_, expected) in enumerate(KNOWN_ANSWERS):
        assert [values[q][0][k] for k in range(len(expected))] == expected


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["tweets", "adversarial", "quirks"])
def test_values_equal_host_slices(gpjson, kind):
    if kind == "tweets":
        data, paths = datagen.tweets(3 << 20, seed=datagen.SEED_BASE + 71).tobytes(), TWEET_PATHS + ["$.user"]
    elif kind == "adversarial":
        data, paths = datagen.adversarial(3 << 20, seed=datagen.SEED_BASE + 72).tobytes(), ADV_PATHS + ["$.arr[0:3]"]
    else:
        # [0] as the last step on an empty array stores (position of ']', -1): unreadable
        data = b'{"a": [], "b": "x\\u00e9\\"y"}\n{"a": [1, 2]}\n\n{"b": "\xc3\xa9t\xc3\xa9"}\n{"a": [ ]}'
        paths = ["$.a[0]", "$.b", "$.a", "$.a[1]"]
    values, result = values_and_result(gpjson, data, paths)
    assert_same(values, result)
    if kind == "quirks":
        assert read(values[0][0], 0)[0] == "unreadable"
        assert values[1][3][0] == "\"été\""
    # the compact buffer holds exactly the present values
    present = values.kinds == gj.VALUE_PRESENT
    lengths = np.diff(values.offsets).reshape(values.kinds.shape)
    assert (lengths[~present] == 0).all()
    assert values.offsets[-1] == len(values.data)


@pytest.mark.gpu
def test_values_device_entry(gpjson):
    """gpj_values_device on caller-owned device buffers, including a byte
    buffer that is too small (GPJ_ELIMIT with the total, kinds and offsets
    complete) and no pairs at all."""
    import ctypes

    import torch

    data = datagen.tweets(1 << 20, seed=datagen.SEED_BASE + 73).tobytes()
    compiled = [gj.compile_path(p) for p in TWEET_PATHS]
    f = gpjson.load_bytes(data)
    lib, h = gpjson._native.lib, gpjson._native.h
    try:
        f.build_index(4)
        pairs = f.run(compiled)
        d_pairs = torch.from_numpy(pairs.reshape(-1)).cuda()
        npairs = pairs.size // 2
        d_kinds = torch.zeros(npairs, dtype=torch.uint8, device="cuda")
        d_off = torch.zeros(npairs + 1, dtype=torch.int64, device="cuda")
        total = ctypes.c_int64()
        rc = lib.gpj_values_device(h, f._h, d_pairs.data_ptr(), npairs, d_kinds.data_ptr(), d_off.data_ptr(), None, 0,
                                   ctypes.byref(total))
        assert rc == gj._lib.GPJ_ELIMIT and total.value > 0
        d_bytes = torch.zeros(total.value, dtype=torch.uint8, device="cuda")
        gpjson._native.check(lib.gpj_values_device(h, f._h, d_pairs.data_ptr(), npairs, d_kinds.data_ptr(),
                                                   d_off.data_ptr(), d_bytes.data_ptr(), total.value,
                                                   ctypes.byref(total)))
        kinds, offs, got = d_kinds.cpu().numpy(), d_off.cpu().numpy(), d_bytes.cpu().numpy().tobytes()
        flat = pairs.reshape(-1, 2)
        want = b"".join(data[s:e] for s, e in flat if s != -1)
        assert got == want
        assert (kinds == np.where(flat[:, 0] == -1, gj.VALUE_NULL, gj.VALUE_PRESENT)).all()
        lens = np.where(flat[:, 0] == -1, 0, flat[:, 1] - flat[:, 0])
        assert np.array_equal(offs, np.concatenate([[0], np.cumsum(lens)]))
        gpjson._native.check(lib.gpj_values_device(h, f._h, None, 0, None, d_off.data_ptr(), None, 0,
                                                   ctypes.byref(total)))
        assert total.value == 0 and int(d_off[0]) == 0
    finally:
        f.release()
