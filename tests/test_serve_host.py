"""Host-side parts of the serving loop (no GPU): request generation,
resident-size accounting and latency statistics."""

from __future__ import annotations

import numpy as np

from gpjson_b200 import serve
from oracle import jsonpath_oracle


def test_path_pool_compiles_within_levels():
    assert len(serve.PATH_POOL) == 32 and len(set(serve.PATH_POOL)) == 32
    depths = [jsonpath_oracle.compile_path(p)[1] for p in serve.PATH_POOL]
    assert max(depths) == serve.POOL_LEVELS and min(depths) == 1


def test_poisson_requests_rate_and_zipf():
    names = [f"c{i}" for i in range(64)]
    reqs = serve.poisson_requests(names, 20000, rate=2000.0, seed=3)
    t = np.array([r.arrival for r in reqs])
    assert t[0] == 0.0 and np.all(np.diff(t) >= 0)
    assert abs(len(reqs) / t[-1] - 2000.0) < 100.0
    counts = np.bincount([names.index(r.corpus) for r in reqs], minlength=64)
    assert counts[0] > counts[1] > counts[10] > 0  # Zipf: the first corpora dominate
    assert all(p in serve.PATH_POOL for r in reqs for p in r.paths)


def test_stats_percentiles():
    s = serve.ServeStats(requests=100, seconds=2.0, latencies_ms=[float(i) for i in range(1, 101)], batches=10)
    d = s.summary()
    assert d["queries_per_s"] == 50.0 and d["mean_batch"] == 10.0
    assert d["p50_ms"] == 51.0 and d["p99_ms"] == 99.0


def test_resident_bytes():
    n = 1 << 20
    assert serve.resident_bytes(n, 6) == n + 8 * (n // 64) * 8 + 8 * (n // 256 + 1024)
