"""GPU parity of batched requests (gpj_batch): many files of uneven size and
shape, several requests per file, each request's results against the
single-file query path and the oracle; a second run on the now-resident
indexes launches only the query kernel."""

from __future__ import annotations

import json
import random

import numpy as np
import pytest

import gpjson_b200 as gj
from gpjson_b200 import datagen
from oracle import oracle

POOL = [
    "$.user.lang", "$.id", "$.user.followers_count", "$.entities.hashtags[0].text", "$.text",
    "$.a.b.c.d", "$.arr[5]", "$.x[0].y[2].z", "$.user", "$.entities.hashtags[1]", "$.k",
]


def pretty(seed: int) -> bytes:
    rng = random.Random(seed)
    doc = [{"k": rng.randint(0, 9), "a": {"b": {"c": {"d": "x\\"}}}, "arr": list(range(rng.randint(0, 9)))}
           for _ in range(40)]
    return json.dumps(doc, indent=2).encode()


def corpus(rng: random.Random):
    files = [
        datagen.tweets(3 << 20, seed=datagen.SEED_BASE + 11).tobytes(),
        datagen.tweets(70 << 10, seed=datagen.SEED_BASE + 12).tobytes(),
        datagen.tweets(5000, seed=datagen.SEED_BASE + 13).tobytes(),
        datagen.adversarial(2 << 20, seed=datagen.SEED_BASE + 14).tobytes(),
        pretty(15),  # not line-delimited: indexed again alone
        b"",
        b'{"k": 1}\n{"k": [2]}\n',
        b'{"k":"' + b"y" * 40000 + b'"}\n{"k": 3}',  # a line longer than the look-ahead
    ]
    requests = []
    for i, _ in enumerate(files):
        for _ in range(rng.randint(1, 3)):
            requests.append((i, rng.sample(POOL, rng.randint(1, 4))))
    return files, requests


@pytest.mark.gpu
def test_batch_matches_single_file_path_and_oracle(gpjson):
    rng = random.Random(5)
    data, requests = corpus(rng)
    files = [gpjson.load_bytes(d) for d in data]
    b = gpjson.batch()
    try:
        items = [b.add(files[i], paths) for i, paths in requests]
        b.run()
        got = [b.result(it) for it in items]
        # a second run reuses the resident indexes: one find_value launch
        # (and the one for lines handed to a warp each)
        before = gpjson.kernel_launches()
        b.run()
        assert gpjson.kernel_launches() - before == (2 if gpjson.tuning()["long_line_bytes"] >= 0 else 1)
        again = [b.result(it) for it in items]
    finally:
        b.release()
        for f in files:
            f.release()
    for (i, paths), g, a in zip(requests, got, again):
        assert np.array_equal(g, a)
        alone = gpjson.load_bytes(data[i])
        try:
            want = alone.query_paths(paths)
        finally:
            alone.release()
        # the batch's slot count is the largest among its file's requests
        assert np.array_equal(g[:, :, : want.shape[2]], want), (i, paths)
        assert (g[:, :, want.shape[2]:] == -1).all()
        ref = oracle.query(data[i], paths)
        assert np.array_equal(want, ref), (i, paths)


@pytest.mark.gpu
def test_batch_errors(gpjson):
    f = gpjson.load_bytes(b'{"a": 1}\n')
    b = gpjson.batch()
    try:
        with pytest.raises(gj.JSONPathException):
            b.add(f, ["$.a", "$$"])
        with pytest.raises(gj.UnsupportedJSONPathException):
            b.add(f, ["$..a"])
        with pytest.raises(gj.GPJSONException):
            b.result(0)
        it = b.add(f, ["$.a"])
        b.run()
        r = b.result(it)
        # two lines: the newline index also counts the empty line after the last '\n'
        assert r.shape == (1, 2, 1, 2) and r[0, 0, 0, 0] == 6 and r[0, 1, 0, 0] == -1
        b.clear()
        assert len(b) == 0
    finally:
        b.release()
        f.release()


@pytest.mark.gpu
def test_batch_replays_its_query_graph(gpjson):
    """A batch run again with the same requests on the same resident indexes
    replays the CUDA graph of its query phase (phase batch_query_replay);
    results are the same; holding a result, adding a request or changing the
    launch shapes makes the next run capture a new graph."""
    rng = random.Random(9)
    data, requests = corpus(rng)
    files = [gpjson.load_bytes(d) for d in data]
    b = gpjson.batch()

    def phases():
        return [p["name"] for p in gpjson.timings()["phases"]]

    try:
        items = [b.add(files[i], paths) for i, paths in requests]
        b.run()  # indexes the files; queries launched directly
        first = [b.result(it).copy() for it in items]
        b.run()  # unchanged: the query phase is captured as a graph and launched
        assert all(np.array_equal(b.result(it), x) for it, x in zip(items, first))
        gpjson._native.lib.gpj_reset_timings(gpjson._native.h)
        b.run()
        assert "batch_query_replay" in phases()
        again = [b.result(it) for it in items]
        assert all(np.array_equal(x, y) for x, y in zip(first, again))
        # a result of the last run is still held: no replay into its buffer
        gpjson._native.lib.gpj_reset_timings(gpjson._native.h)
        b.run()
        assert "batch_query_replay" not in phases() and "batch_query" in phases()
        b.run()  # captured again, into another buffer
        held = [b.result(it) for it in items]
        assert all(np.array_equal(x, y) for x, y in zip(first, held))
        del again, held
        gpjson._native.lib.gpj_reset_timings(gpjson._native.h)
        b.run()
        assert "batch_query_replay" in phases()
        gpjson.set_tuning(query_ctas_per_sm=1)
        gpjson._native.lib.gpj_reset_timings(gpjson._native.h)
        b.run()
        assert "batch_query_replay" not in phases()
        gpjson.set_tuning(query_ctas_per_sm=0)
        b.add(files[0], ["$.id"])
        gpjson._native.lib.gpj_reset_timings(gpjson._native.h)
        b.run()
        assert "batch_query_replay" not in phases()
        assert all(np.array_equal(b.result(it), x) for it, x in zip(items, first))
    finally:
        gpjson.set_tuning(query_ctas_per_sm=0)
        b.release()
        for f in files:
            f.release()
