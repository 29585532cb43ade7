"""GPU parity at the sizes the throughput numbers are quoted on, against the
OpenMP oracle (64-bit offsets, Sequential.java:14-344):

- tweet-like NDJSON of 2 GiB + 64 MiB, so that lines and values lie past
  byte 2^31 and one line straddles it (the reference's int offsets overflow
  there): newline index, string index, 4 leveled bitmaps and the 4 queries,
  through the resident-index path and the pipelined loader;
- the adversarial generator at 4 GiB (lines to 1 MiB, nesting to 16,
  backslash runs) with its three queries;
- a line longer than 2^31 bytes, so the interpreter's 32-bit line-relative
  positions cannot hold it and the 64-bit interpreter runs on the GPU, and a
  whitespace skip from a short line across a 2 GiB run of spaces (the
  32-bit pass stops at its limit and the line is evaluated again in 64 bits).
"""

from __future__ import annotations

import numpy as np
import pytest

import gpjson_b200 as gj
from gpjson_b200 import datagen
from oracle import oracle

TWEET_PATHS = ["$.user.lang", "$.id", "$.user.followers_count", "$.entities.hashtags[0].text"]
ADV_PATHS = ["$.a.b.c.d", "$.arr[5]", "$.x[0].y[2].z"]
TWO_GIB = 1 << 31


def _index_equal(f: gj.File, want: oracle.Index, levels: int) -> None:
    assert np.array_equal(f.newline_index(), want.newlines), "newline index"
    assert np.array_equal(f.string_index(), want.strings), "string index"
    assert np.array_equal(f.leveled_bitmaps(levels), want.levels), "leveled bitmaps"


@pytest.mark.gpu
def test_tweets_past_two_gib(gpjson):
    data = datagen.tweets(TWO_GIB + (64 << 20), seed=datagen.SEED_BASE + 1, p_empty_hashtags=0.3)
    want_idx = oracle.Index(data, 4, mt=True)
    nl = want_idx.newlines
    k = int(np.searchsorted(nl, TWO_GIB, side="right")) - 1
    assert nl[k] < TWO_GIB < nl[k + 1], "a line straddles byte 2^31"
    want = oracle.query(data, TWEET_PATHS, mt=True, index=want_idx)
    assert (want[:, :, 0, 0] >= TWO_GIB).sum() > 100_000, "values past byte 2^31"
    compiled = [gj.compile_path(p) for p in TWEET_PATHS]
    f = gpjson.load_bytes(data)
    try:
        f.build_index(4)
        _index_equal(f, want_idx, 4)
        assert np.array_equal(f.run(compiled), want), "queries on the resident index"
    finally:
        f.release()
    f = gpjson.load_bytes(data)
    try:
        assert np.array_equal(f.query_paths(TWEET_PATHS), want), "gpj_query_paths"
    finally:
        f.release()
    f, got = gpjson.load_bytes_query(data, 4, compiled)
    try:
        assert np.array_equal(got, want), "pipelined copy + index + queries"
        _index_equal(f, want_idx, 4)
    finally:
        f.release()


@pytest.mark.gpu
def test_adversarial_four_gib(gpjson):
    data = datagen.adversarial(4 << 30, seed=datagen.SEED_BASE + 2)
    compiled = [gj.compile_path(p) for p in ADV_PATHS]
    levels = max(c.max_depth for c in compiled)
    want_idx = oracle.Index(data, levels, mt=True)
    want = oracle.query(data, ADV_PATHS, mt=True, index=want_idx)
    hits = (want[:, :, 0, 0] >= 0).sum(axis=1)
    lines = want.shape[1]
    assert all(0.3 * lines < h < 0.95 * lines for h in hits), hits
    f = gpjson.load_bytes(data)
    try:
        assert np.array_equal(f.query_paths(ADV_PATHS), want), "gpj_query_paths"
        _index_equal(f, want_idx, levels)
    finally:
        f.release()
    f, got = gpjson.load_bytes_query(data, levels, compiled)
    try:
        assert np.array_equal(got, want), "pipelined copy + index + queries"
    finally:
        f.release()


def _bytes(*parts) -> np.ndarray:
    """Concatenates byte strings and (byte value, count) runs into one array."""
    size = sum(len(p) if isinstance(p, bytes) else p[1] for p in parts)
    out = np.empty(size, dtype=np.uint8)
    pos = 0
    for p in parts:
        if isinstance(p, bytes):
            out[pos:pos + len(p)] = np.frombuffer(p, dtype=np.uint8)
            pos += len(p)
        else:
            out[pos:pos + p[1]] = p[0]
            pos += p[1]
    return out


def _check_against_oracle(gpjson, data: np.ndarray, paths: list[str]) -> np.ndarray:
    compiled = [gj.compile_path(p) for p in paths]
    levels = max(c.max_depth for c in compiled)
    want_idx = oracle.Index(data, levels, mt=True)
    want = oracle.query(data, paths, mt=True, index=want_idx)
    f = gpjson.load_bytes(data)
    try:
        f.build_index(levels)
        _index_equal(f, want_idx, levels)
        got = f.run(compiled)
    finally:
        f.release()
    assert np.array_equal(got, want)
    return got


@pytest.mark.gpu
def test_line_longer_than_two_gib(gpjson):
    # line 1 holds a string of 2^31 bytes; its later values lie past 2^31 from the line start
    data = _bytes(b'{"a":{"b":1},"t":[0]}\n{"s":"', (ord("x"), TWO_GIB),
                  b'","a":{"b":2},"t":[1,2,3],"u":"\\"x"}\n{"a":{"b":3}}')
    got = _check_against_oracle(gpjson, data, ["$.a.b", "$.t[1]", "$.s", "$.u"])
    assert got[0, 1, 0, 0] > TWO_GIB and got[1, 1, 0, 0] > TWO_GIB and got[3, 1, 0, 0] > TWO_GIB
    assert got[2, 1, 0, 1] - got[2, 1, 0, 0] == TWO_GIB + 2


@pytest.mark.gpu
def test_whitespace_skip_past_two_gib(gpjson):
    # "$[0]" on line 0 stores after a skip over its '\n' and 2^31 spaces of line 1
    data = _bytes(b"[\n", (ord(" "), TWO_GIB), b'1]\n{"a":[5]}')
    got = _check_against_oracle(gpjson, data, ["$[0]", "$.a[0]"])
    assert got[0, 0, 0, 0] == TWO_GIB + 2
