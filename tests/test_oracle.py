"""Pins the oracle to the reference's own known answers and fixture-derived
expectations, and checks its multi-threaded variants."""

from __future__ import annotations

import json

import numpy as np
import pytest

from gpjson_b200 import datagen
from oracle import oracle
from tests.conftest import GOLDEN, fixture_bytes

SIMPLE = "query_gpu_function/simple_single_line.ldjson"
NOT_FOUND = "query_gpu_function/not_found_in_current_level.ldjson"

# QueryFunctionTest.java:86-167: (path, values over all lines and slots)
KNOWN_ANSWERS = [
    ("$.user.lang", ['"nl"']),  # :86-92
    ("$.user.id", ["8723"]),  # :94-100
    ("$.user.foo", [None]),  # :102-108
    ("$.apple.lang", [None]),  # :110-116
    ("$.user.values[0]", ['"12"']),  # :118-124
    ("$.user.values[2]", ["14"]),  # :126-132
    ("$.user.values[8]", [None]),  # :134-140
    ("$.user.values[0:3]", ['"12"', '"13"', "14"]),  # :142-150
    ("$.user.values[2:4]", ["14", '"15"']),  # :152-159
    ("$.user.lang[?(@ == 'nl')]", ['"nl"']),  # :161-167
]


def values(data: bytes, offsets: np.ndarray) -> list:
    """resultToValues (QueryFunctionTest.java:212-230) over ResultItem
    semantics (ResultItem.java:32-52)."""
    out = []
    for start, end in offsets.reshape(-1, 2):
        out.append(None if start == -1 else data[start:end].decode("utf-8"))
    return out


@pytest.mark.parametrize("path,expected", KNOWN_ANSWERS, ids=[k[0] for k in KNOWN_ANSWERS])
def test_known_answers(path, expected):
    data = fixture_bytes(SIMPLE)
    assert values(data, oracle.query(data, [path])) == expected


def test_key_not_found_in_current_level():
    # QueryFunctionTest.java:169-198: $.a.a has no non-null value
    data = fixture_bytes(NOT_FOUND)
    assert all(v is None for v in values(data, oracle.query(data, ["$.a.a"])))


def _expected_escape_and_quote(data: bytes):
    """StringIndexTest.createExpectedEscapeIndex / createExpectedQuoteIndex
    (:388-426), an independent restatement of the escape rule."""
    words = (len(data) + 63) // 64
    esc = np.zeros(words, dtype=np.uint64)
    quote = np.zeros(words, dtype=np.uint64)
    carry = 0
    for i, c in enumerate(data):
        if carry == 1:
            esc[i // 64] |= np.uint64(1 << (i % 64))
        if c == ord('"') and carry != 1:
            quote[i // 64] |= np.uint64(1 << (i % 64))
        carry = (carry ^ 1) if c == ord("\\") else 0
    return esc, quote


@pytest.mark.parametrize("name", ["simple", "escape_carry", "very_long_string"])
def test_string_index_matches_quote_prefix_xor(name):
    data = fixture_bytes(f"stages/string_index/{name}.txt")
    _, quote = _expected_escape_and_quote(data)
    want = np.zeros_like(quote)
    inside = 0
    for w in range(len(quote)):
        x = int(quote[w])
        acc = 0
        for b in range(64):
            if (x >> b) & 1:
                inside ^= 1
            if inside and w * 64 + b < len(data):
                acc |= 1 << b
        want[w] = acc
    assert np.array_equal(oracle.string_index(data), want)


@pytest.mark.parametrize("name", ["even_positions", "odd_positions", "random_data", "aligned_random_data"])
def test_newline_index_fixtures(name):
    # NewlineIndexTest.createExpectedIndex = Sequential.createNewlineIndex
    data = fixture_bytes(f"stages/newline_index/{name}.txt")
    nl = oracle.newline_index(data)
    assert nl[0] == 0
    assert np.array_equal(nl[1:], np.flatnonzero(np.frombuffer(data, np.uint8) == 10))


def test_leveled_bitmaps_simple_fixture_by_hand():
    # stages/leveled_bitmaps_index/simple.json: the brackets inside strings are
    # not structural; ':' ',' of the object at level 0, the array at level 1.
    data = fixture_bytes("stages/leveled_bitmaps_index/simple.json")
    idx = oracle.Index(data, 16)
    lv0 = [i for i in range(len(data)) if (int(idx.levels[0][i // 64]) >> (i % 64)) & 1]
    lv1 = [i for i in range(len(data)) if (int(idx.levels[1][i // 64]) >> (i % 64)) & 1]
    text = data.decode()
    assert [text[i] for i in lv0] == ["{", ":", ",", ":", ",", ":", "}"]
    assert [text[i] for i in lv1] == ["[", ",", "]"]
    assert not idx.levels[2:].any()


def test_golden_expectations_reproduce():
    expected = json.loads((GOLDEN / "expected.json").read_text())
    import hashlib

    for rel, e in expected.items():
        data = fixture_bytes(rel)
        assert hashlib.sha256(data).hexdigest() == e["sha256"], rel
        idx = oracle.Index(data, 16)
        assert hashlib.sha256(idx.newlines.tobytes()).hexdigest() == e["newline_sha256"], rel
        assert hashlib.sha256(idx.strings.tobytes()).hexdigest() == e["string_sha256"], rel
        assert hashlib.sha256(idx.levels.tobytes()).hexdigest() == e["levels16_sha256"], rel


@pytest.mark.parametrize("gen", ["tweets", "adversarial"])
def test_multithreaded_oracle_equals_sequential(gen):
    data = (datagen.tweets(3 << 20) if gen == "tweets" else datagen.adversarial(6 << 20)).tobytes()
    paths = (
        ["$.user.lang", "$.id", "$.entities.hashtags[0].text"]
        if gen == "tweets"
        else ["$.a.b.c.d", "$.arr[5]", "$.x[0].y[2].z"]
    )
    a = oracle.Index(data, 5)
    b = oracle.Index(data, 5, mt=True)
    assert np.array_equal(a.newlines, b.newlines)
    assert np.array_equal(a.strings, b.strings)
    assert np.array_equal(a.levels, b.levels)
    assert np.array_equal(oracle.query(data, paths, index=a), oracle.query(data, paths, mt=True, index=b))


def test_generators_hit_the_stated_miss_rates():
    data = datagen.tweets(4 << 20).tobytes()
    r = oracle.query(data, ["$.entities.hashtags[0].text", "$.user.lang"])
    lines = r.shape[1]
    miss_hashtag = np.mean(r[0, :, 0, 0] == -1)
    miss_lang = np.mean(r[1, :, 0, 0] == -1)
    assert 0.25 < miss_hashtag < 0.40  # 30% empty arrays (+ block padding lines)
    assert miss_lang < 0.05 and lines > 1000
    adv = datagen.adversarial(16 << 20).tobytes()
    r = oracle.query(adv, ["$.a.b.c.d", "$.arr[5]", "$.x[0].y[2].z"])
    real = r.shape[1]
    for q in range(3):
        miss = np.mean(r[q, :, 0, 0] == -1)
        assert 0.08 < miss < 0.6, (q, miss, real)
