"""The serving loop on the GPU: every request's result is the same in the
continuous-batching mix as alone, and equals the oracle's; corpora are
loaded on demand and evicted (least recently used) under the budget."""

from __future__ import annotations

import numpy as np
import pytest

from gpjson_b200 import datagen, serve
from oracle import oracle


def corpora() -> dict[str, np.ndarray]:
    out = {}
    for i, size in enumerate([64 << 10, 300 << 10, 1 << 20, 3 << 20]):
        out[f"tweets{i}"] = datagen.tweets(size, seed=datagen.SEED_BASE + 40 + i)
    for i, size in enumerate([700 << 10, 2 << 20]):
        out[f"adv{i}"] = datagen.adversarial(size, seed=datagen.SEED_BASE + 50 + i)
    return out


def check_results(reqs, data, want_cache):
    for r in reqs:
        key = (r.corpus, tuple(r.paths))
        if key not in want_cache:
            want_cache[key] = oracle.query(data[r.corpus].tobytes(), list(r.paths))
        want = want_cache[key]
        got = r.result
        assert got.shape[:2] == want.shape[:2], key
        assert np.array_equal(got[:, :, : want.shape[2]], want), key
        assert (got[:, :, want.shape[2]:] == -1).all(), key


@pytest.mark.gpu
def test_serving_mix_equals_alone_and_oracle():
    data = corpora()
    names = list(data)
    # room for about half of the corpora: loads and evictions happen while serving
    budget = sum(serve.resident_bytes(data[n].size) for n in names) // 2
    budget = max(budget, max(serve.resident_bytes(d.size) for d in data.values()) * 2)
    reqs = serve.poisson_requests(names, 240, rate=4000.0, paths_per_request=2, seed=7)
    alone = [serve.Request(r.arrival, r.corpus, list(r.paths)) for r in reqs[:40]]
    srv = serve.Server(data, budget_bytes=budget)
    try:
        stats = srv.serve(reqs, keep_results=True)
        solo = srv.serve(alone, per_request=True, keep_results=True)
    finally:
        srv.close()
    cache = {}
    check_results(reqs, data, cache)
    check_results(alone, data, cache)
    for a, r in zip(alone, reqs[:40]):
        w = min(a.result.shape[2], r.result.shape[2])
        assert np.array_equal(a.result[:, :, :w], r.result[:, :, :w])
    s = stats.summary()
    assert s["requests"] == 240 and s["batches"] < 240  # requests were batched
    assert s["loads"] >= len(names) and s["evictions"] > 0
    assert 0 <= s["p50_ms"] <= s["p99_ms"]
    assert solo.summary()["batches"] == 40
