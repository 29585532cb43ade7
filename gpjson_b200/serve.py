"""Serving: (corpus, JSONPath) requests against resident corpora, over the
native request server (gpj_serve_*, include/gpjson_b200.h).

The server keeps corpora resident in device memory with their structural
indexes under a byte budget (least recently used out, an evicted corpus's
bytes counting until its memory is released), loads cold ones from
page-locked host memory on a loader thread, and batches continuously:
each of its serving threads takes every arrived request whose corpus is
resident and evaluates them in one batch on its own stream, so iterations
overlap on the device.  This module paces requests by their arrival times,
collects the results and computes latency statistics.  The per-request form
(one request at a time) is the baseline the batched form is measured
against.

The reference has no serving mode; its query() reads, indexes and queries
the file on every call (functions/QueryFunction.java:48-265).
"""

from __future__ import annotations

import ctypes
import json
import statistics
import time
from ctypes import byref, c_char_p, c_int, c_int64, c_size_t, c_uint64, c_void_p
from dataclasses import dataclass, field

import numpy as np

from . import _lib, _result_array

# 32 paths of depth 1-6 over the two synthetic schemas (tweet-like objects;
# the adversarial generator's a/b/c/d chains, arrays and x/y/z nesting),
# mixing field and index steps.
PATH_POOL = [
    "$.id", "$.text", "$.user", "$.entities",
    "$.user.lang", "$.user.id", "$.user.name", "$.user.followers_count",
    "$.entities.hashtags", "$.entities.hashtags[0]", "$.entities.hashtags[1]", "$.entities.hashtags[2]",
    "$.entities.hashtags[0].text", "$.entities.hashtags[1].text", "$.entities.hashtags[4].text",
    "$.user.lang[?(@ == 'en')]",
    "$.a", "$.a.b", "$.a.b.c", "$.a.b.c.d", "$.a.b.c.d.e", "$.a.b.c.d.e.f",
    "$.arr", "$.arr[0]", "$.arr[5]", "$.arr[100]", "$.arr[0:3]",
    "$.x[0]", "$.x[0].y", "$.x[0].y[2]", "$.x[0].y[2].z", "$.x[1].y[0].z",
]
POOL_LEVELS = 6  # every pool path needs at most 6 levels


def resident_bytes(n: int, levels: int = POOL_LEVELS) -> int:
    """Device bytes of a resident corpus: input, string index, ':' bitmap,
    leveled bitmaps and a newline-index allowance."""
    words = (n + 63) // 64
    return n + 8 * words * (2 + levels) + 8 * (n // 256 + 1024)


@dataclass
class Request:
    arrival: float  # seconds after the start of serve()
    corpus: str
    paths: list[str]
    done: float = -1.0
    result: np.ndarray | None = None


@dataclass
class ServeStats:
    requests: int
    seconds: float
    latencies_ms: list[float] = field(repr=False)
    batches: int = 0
    loads: int = 0
    evictions: int = 0

    @property
    def queries_per_s(self) -> float:
        return self.requests / self.seconds if self.seconds > 0 else 0.0

    def percentile(self, q: float) -> float:
        xs = sorted(self.latencies_ms)
        if not xs:
            return 0.0
        k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
        return xs[k]

    def summary(self) -> dict:
        return {
            "requests": self.requests,
            "seconds": round(self.seconds, 4),
            "queries_per_s": round(self.queries_per_s, 1),
            "p50_ms": round(self.percentile(50), 3),
            "p99_ms": round(self.percentile(99), 3),
            "mean_ms": round(statistics.mean(self.latencies_ms), 3) if self.latencies_ms else 0.0,
            "batches": self.batches,
            "mean_batch": round(self.requests / self.batches, 2) if self.batches else 0.0,
            "loads": self.loads,
            "evictions": self.evictions,
        }


class ServerError(RuntimeError):
    def __init__(self, message: str, code: int):
        super().__init__(message)
        self.code = code


class Server:
    """Resident corpora under `budget_bytes` and continuous batching, on the
    native server (`workers` serving threads, each its own stream)."""

    def __init__(self, corpora: dict[str, np.ndarray], budget_bytes: int, device: int = 0,
                 levels: int = POOL_LEVELS, max_batch: int = 512, workers: int = 2):
        self.lib = _lib.load()
        self.max_batch = max_batch
        self.workers = workers
        cfg = _lib.ServerConfig(device, levels, int(budget_bytes), max_batch, workers)
        self._h = c_void_p()
        self._check(self.lib.gpj_serve_create(byref(cfg), byref(self._h)), "gpj_serve_create")
        self._arrays = {}
        self._ids: dict[str, int] = {}
        for name, arr in corpora.items():
            a = np.ascontiguousarray(arr, dtype=np.uint8)
            cid = c_int()
            self._check(self.lib.gpj_serve_add_corpus(self._h, a.ctypes.data, a.size, byref(cid)),
                        f"gpj_serve_add_corpus({name})")
            self._arrays[name] = a  # must outlive the server
            self._ids[name] = cid.value

    @staticmethod
    def _check(rc: int, what: str) -> None:
        if rc != _lib.GPJ_OK:
            raise ServerError(f"{what} failed ({rc})", rc)

    def stats(self) -> dict:
        n = c_size_t()
        self.lib.gpj_serve_stats(self._h, None, 0, byref(n))
        buf = ctypes.create_string_buffer(n.value + 1)
        self._check(self.lib.gpj_serve_stats(self._h, buf, n.value + 1, byref(n)), "gpj_serve_stats")
        return json.loads(buf.value.decode())

    def serve(self, requests: list[Request], per_request: bool = False, keep_results: bool = False) -> ServeStats:
        """Submits `requests` at their arrival times (seconds from now) and
        waits for all; per_request=True runs one request at a time (the
        baseline form).  Latency = completion - arrival."""
        lib = self.lib
        reqs = sorted(requests, key=lambda r: r.arrival)
        if per_request:
            self._check(lib.gpj_serve_set_batching(self._h, 1, 1), "gpj_serve_set_batching")
        else:
            self._check(lib.gpj_serve_set_batching(self._h, self.max_batch, self.workers), "gpj_serve_set_batching")
        before = self.stats()
        ids: list[int] = []
        t0_ns = lib.gpj_serve_now_ns(self._h)
        t0 = time.perf_counter()
        collected = 0

        def collect(timeout_ms: int) -> bool:
            """Takes the oldest outstanding request's result if it is done
            (results are handed back as they finish, so their memory is
            released early)."""
            nonlocal collected
            r, rid = reqs[collected], ids[collected]
            res, sub, done = c_void_p(), c_int64(), c_int64()
            rc = lib.gpj_serve_poll(self._h, rid, timeout_ms, byref(res), byref(sub), byref(done))
            if rc == _lib.GPJ_EAGAIN:
                return False
            if rc != _lib.GPJ_OK:
                if res.value:
                    lib.gpj_result_release(res)
                raise ServerError(f"request for {r.corpus} {r.paths} failed ({rc})", rc)
            r.done = (done.value - t0_ns) / 1e9
            if keep_results:
                r.result = _result_array(lib, res)
            else:
                lib.gpj_result_release(res)
            collected += 1
            return True

        for r in reqs:
            while True:
                wait = r.arrival - (time.perf_counter() - t0)
                if wait <= 0:
                    break
                if collected < len(ids) and collect(0):
                    continue
                time.sleep(min(wait, 0.0005))
            arr = (c_char_p * len(r.paths))(*[p.encode("utf-8") for p in r.paths])
            rid = c_uint64()
            self._check(lib.gpj_serve_submit(self._h, self._ids[r.corpus], len(r.paths), arr, byref(rid)),
                        "gpj_serve_submit")
            ids.append(rid.value)
        while collected < len(ids):
            collect(-1)
        after = self.stats()
        last = max(r.done for r in reqs) if reqs else 0.0
        first = min(r.arrival for r in reqs) if reqs else 0.0
        return ServeStats(
            requests=len(reqs), seconds=last - first,
            latencies_ms=[1000.0 * (r.done - r.arrival) for r in reqs],
            batches=after["batches"] - before["batches"], loads=after["loads"], evictions=after["evictions"],
        )

    def close(self) -> None:
        if self._h:
            self.lib.gpj_serve_destroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_requests(corpora: list[str], count: int, rate: float, zipf_s: float = 1.1, paths_per_request: int = 1,
                     seed: int = 0x67706A73 + 4) -> list[Request]:
    """Poisson arrivals at `rate` per second, corpus popularity Zipf(s) over
    `corpora` (in the given order), paths drawn from PATH_POOL."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    arrivals = np.cumsum(gaps) - gaps[0]
    ranks = np.arange(1, len(corpora) + 1, dtype=np.float64)
    weights = ranks ** -zipf_s
    weights /= weights.sum()
    picks = rng.choice(len(corpora), size=count, p=weights)
    out = []
    for t, c in zip(arrivals, picks):
        paths = [PATH_POOL[i] for i in rng.choice(len(PATH_POOL), size=paths_per_request, replace=False)]
        out.append(Request(arrival=float(t), corpus=corpora[c], paths=paths))
    return out
