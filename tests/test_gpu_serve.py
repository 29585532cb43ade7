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


@pytest.mark.gpu
def test_server_through_the_c_abi_from_two_threads():
    """gpj_serve_* called directly: two client threads submit requests for
    two corpora at once, each result (gpj_result, its own slots) equals the
    oracle's; a path deeper than the server's levels and a bad corpus are
    refused; GPJ_EAGAIN until a request is done."""
    import ctypes
    import threading
    from ctypes import byref, c_char_p, c_int, c_int64, c_uint64, c_void_p

    from gpjson_b200 import _lib, _result_array

    lib = _lib.load()
    data = {"t": datagen.tweets(2 << 20, seed=datagen.SEED_BASE + 60),
            "a": datagen.adversarial(3 << 20, seed=datagen.SEED_BASE + 61)}
    cfg = _lib.ServerConfig(0, 5, 1 << 30, 64, 2)
    h = c_void_p()
    assert lib.gpj_serve_create(byref(cfg), byref(h)) == _lib.GPJ_OK
    try:
        ids = {}
        for name, arr in data.items():
            cid = c_int()
            assert lib.gpj_serve_add_corpus(h, arr.ctypes.data, arr.size, byref(cid)) == _lib.GPJ_OK
            ids[name] = cid.value
        jobs = [("t", ["$.user.lang", "$.entities.hashtags[0:2]"]), ("a", ["$.arr[5]"]), ("t", ["$.id"]),
                ("a", ["$.a.b.c.d", "$.x[0].y[2].z"])] * 6
        out = [None] * len(jobs)

        def client(k0):
            for k in range(k0, len(jobs), 2):
                name, paths = jobs[k]
                arr = (c_char_p * len(paths))(*[p.encode() for p in paths])
                rid = c_uint64()
                assert lib.gpj_serve_submit(h, ids[name], len(paths), arr, byref(rid)) == _lib.GPJ_OK
                res, sub, done = c_void_p(), c_int64(), c_int64()
                rc = lib.gpj_serve_poll(h, rid, 0, byref(res), byref(sub), byref(done))
                while rc == _lib.GPJ_EAGAIN:
                    rc = lib.gpj_serve_poll(h, rid, 50, byref(res), byref(sub), byref(done))
                assert rc == _lib.GPJ_OK
                assert 0 <= sub.value <= done.value
                out[k] = _result_array(lib, res)

        threads = [threading.Thread(target=client, args=(i,)) for i in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for (name, paths), got in zip(jobs, out):
            want = oracle.query(data[name].tobytes(), paths)
            assert np.array_equal(got, want), (name, paths)
        deep = (c_char_p * 1)(b"$.a.b.c.d.e.f")
        rid = c_uint64()
        assert lib.gpj_serve_submit(h, ids["a"], 1, deep, byref(rid)) == _lib.GPJ_ELIMIT
        assert lib.gpj_serve_submit(h, 99, 1, deep, byref(rid)) in (_lib.GPJ_EINVAL, _lib.GPJ_ELIMIT)
        n = ctypes.c_size_t()
        buf = ctypes.create_string_buffer(4096)
        assert lib.gpj_serve_stats(h, buf, 4096, byref(n)) == _lib.GPJ_OK
        import json

        st = json.loads(buf.value.decode())
        assert st["served"] == len(jobs) and st["loads"] == 2 and st["batches"] <= len(jobs)
    finally:
        lib.gpj_serve_destroy(h)
