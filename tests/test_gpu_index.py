"""GPU parity of the index kernel against the oracle: the reference's stage
fixtures (StringIndexTest, NewlineIndexTest, LeveledBitmapsIndexTest run on
CombinedIndex/LeveledBitmapsIndex; here the single-pass kernel), random
inputs with strings, escapes and brackets across 64-byte words and 16 KiB
tiles, generated NDJSON of the benchmark shapes, and the device-pointer
entry point."""

from __future__ import annotations

import json
import random

import numpy as np
import pytest

from gpjson_b200 import datagen
from oracle import oracle
from tests.conftest import GOLDEN, fixture_bytes

FIXTURE_NAMES = sorted(json.loads((GOLDEN / "expected.json").read_text()).keys())


def adversarial_bytes(n: int, seed: int = datagen.SEED_BASE + 2) -> bytes:
    return datagen.adversarial(n, seed=seed).tobytes()


def gpu_index(gpjson, data: bytes, levels: int):
    f = gpjson.load_bytes(data)
    try:
        f.build_index(levels)
        return f.newline_index(), f.string_index(), f.leveled_bitmaps(levels)
    finally:
        f.release()


def assert_index_equal(gpjson, data: bytes, levels: int):
    want = oracle.Index(data, levels)
    nl, st, lv = gpu_index(gpjson, data, levels)
    assert np.array_equal(nl, want.newlines), "newline index"
    assert np.array_equal(st, want.strings), "string index"
    assert np.array_equal(lv, want.levels), "leveled bitmaps"


@pytest.mark.gpu
@pytest.mark.parametrize("rel", FIXTURE_NAMES)
def test_reference_fixtures(gpjson, rel):
    expected = json.loads((GOLDEN / "expected.json").read_text())[rel]
    data = fixture_bytes(rel)
    nl, st, lv = gpu_index(gpjson, data, 16)
    import hashlib

    assert hashlib.sha256(nl.tobytes()).hexdigest() == expected["newline_sha256"]
    assert hashlib.sha256(st.tobytes()).hexdigest() == expected["string_sha256"]
    assert hashlib.sha256(lv.tobytes()).hexdigest() == expected["levels16_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(8))
def test_random_bytes(gpjson, seed):
    rng = random.Random(100 + seed)
    alphabet = b'{}[]:,"\\\n ab' if seed % 2 else b'\\\\\\"\n{}[]:,a '
    for n in [0, 1, 15, 16, 17, 63, 64, 65, 16383, 16384, 16385, 70001]:
        data = bytes(rng.choice(alphabet) for _ in range(n))
        assert_index_equal(gpjson, data, rng.choice([1, 2, 4, 5, 8, 9, 16]))


@pytest.mark.gpu
def test_escape_runs_across_tiles(gpjson):
    for run in range(1, 9):
        for shift in (-2, -1, 0, 1, 2):
            pre = b"a" * (3 * 16384 - run + shift)
            data = pre + b"\\" * run + b'"x"{"k":[1,2]}\n' + b"y" * 100
            assert_index_equal(gpjson, data, 3)


@pytest.mark.gpu
def test_backslash_runs_longer_than_many_tiles(gpjson):
    """Backslash runs of 100 KB and more cross several tiles of the exact
    kernel (which resolves the escape state at a tile start by scanning back
    over the run, however long); even and odd lengths, in a line of a
    well-formed file and in pretty-printed input."""
    for run in (100_000, 100_001, 300_003):
        for pre in (0, 5, 16384 - 7):
            line = b'{"s":"' + b"a" * pre + b"\\" * run + b'"x", "t":[1,{"u":"\\\\"}]}'
            assert_index_equal(gpjson, line + b"\n" + b'{"a":[1]}\n' + line, 4)
            assert_index_equal(gpjson, b'{\n "x": [\n  ' + line + b"\n ]\n}\n", 4)


@pytest.mark.gpu
def test_long_string_over_many_tiles(gpjson):
    body = b'{"s":"' + (b"ab\\\"c{[:,]}" * 20000) + b'","t":[1,{"u":2}]}\n'
    assert_index_equal(gpjson, body * 3, 4)


@pytest.mark.gpu
def test_many_short_lines_grow_newline_index(gpjson):
    data = b"\n" * 300000 + b"{}\n" * 1000
    assert_index_equal(gpjson, data, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("levels", [1, 4, 16])
def test_generated_tweets(gpjson, levels):
    assert_index_equal(gpjson, datagen.tweets(24 << 20).tobytes(), levels)


@pytest.mark.gpu
def test_generated_adversarial(gpjson):
    assert_index_equal(gpjson, adversarial_bytes(40 << 20), 16)


@pytest.mark.gpu
def test_device_pointer_entry(gpjson):
    import ctypes

    import torch

    data = datagen.tweets(4 << 20).tobytes()
    n = len(data)
    levels = 4
    words = (n + 63) // 64
    d_file = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
    d_str = torch.empty(words, dtype=torch.int64, device="cuda")
    d_lvl = torch.empty(words * levels, dtype=torch.int64, device="cuda")
    d_nl = torch.empty(n // 64 + 16, dtype=torch.int64, device="cuda")
    lines = ctypes.c_int64()
    lib = gpjson._native.lib
    torch.cuda.synchronize()
    rc = lib.gpj_build_index_device(
        gpjson._native.h, d_file.data_ptr(), n, levels, d_str.data_ptr(), d_lvl.data_ptr(), d_nl.data_ptr(),
        d_nl.numel(), ctypes.byref(lines),
    )
    gpjson._native.check(rc)
    want = oracle.Index(data, levels)
    assert lines.value == len(want.newlines)
    assert np.array_equal(d_nl[: lines.value].cpu().numpy(), want.newlines)
    assert np.array_equal(d_str.cpu().numpy().view(np.uint64), want.strings)
    assert np.array_equal(d_lvl.cpu().numpy().view(np.uint64).reshape(levels, words), want.levels)


@pytest.mark.gpu
def test_index_is_repeatable(gpjson):
    data = datagen.tweets(8 << 20).tobytes()
    f = gpjson.load_bytes(data)
    try:
        f.build_index(4)
        first = (f.newline_index(), f.string_index(), f.leveled_bitmaps(4))
        for _ in range(3):
            f.build_index(4)
            again = (f.newline_index(), f.string_index(), f.leveled_bitmaps(4))
            assert all(np.array_equal(a, b) for a, b in zip(first, again))
    finally:
        f.release()


def indexes_of(f, levels):
    return f.newline_index(), f.string_index(), f.leveled_bitmaps(levels)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ndjson", "long_line", "newline_in_string"])
def test_pipelined_load_and_index(gpjson, case):
    """gpj_file_from_host_indexed (56 MiB chunks copied while earlier chunks
    are indexed) equals the plain copy + index build, including inputs that
    need the rebuild: a line longer than a chunk, a raw newline in a string."""
    base = datagen.tweets(150 << 20)
    if case == "ndjson":
        data = base
    else:
        cut = int(np.flatnonzero(base[100 << 20:] == 10)[0]) + (100 << 20)
        if case == "long_line":
            extra = b'{"k":"' + b"x" * (70 << 20) + b'"}'
        else:
            extra = b'{"k": "a' + bytes([10]) + b'b"}'
        data = np.concatenate([base[: cut + 1], np.frombuffer(extra + b"\n", dtype=np.uint8), base[cut + 1:]])
    levels = 4
    f = gpjson.load_bytes(data)
    g = gpjson.load_bytes_indexed(data, levels)
    try:
        f.build_index(levels)
        want = indexes_of(f, levels)
        got = indexes_of(g, levels)
        for a, b, what in zip(got, want, ("newlines", "strings", "levels")):
            assert np.array_equal(a, b), what
    finally:
        f.release()
        g.release()
    if case == "ndjson":
        ref = oracle.Index(data[: 8 << 20].tobytes(), levels)
        assert np.array_equal(want[0][: len(ref.newlines)], ref.newlines)
