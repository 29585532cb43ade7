"""Serving loop: (corpus, JSONPath) requests against resident corpora.

Each corpus is loaded once (pipelined host copy + index build,
gpj_file_from_host_indexed) and kept in device memory with its structural
index under a byte budget; when a new corpus does not fit, the least
recently used ones not needed by the current requests are released.  Loads
run on a context of their own in a loader thread, so they overlap the
queries running on the serving context.

Continuous batching: every iteration takes all requests that have arrived
and whose corpus is resident and evaluates them in one gpj_batch_run (one
find_value launch over every line of every corpus involved, one copy of the
results); requests arriving meanwhile, or waiting for their corpus to load,
join a later iteration.  The per-request form (one request per run) is the
baseline the batched form is measured against.

The reference has no serving mode; its query() reads, indexes and queries
the file on every call (functions/QueryFunction.java:48-265).
"""

from __future__ import annotations

import collections
import queue
import statistics
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import GPJSON, File

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


class Server:
    """Resident corpora under `budget_bytes` and a continuous-batching loop."""

    def __init__(self, corpora: dict[str, np.ndarray], budget_bytes: int, device: int = 0,
                 levels: int = POOL_LEVELS, max_batch: int = 512):
        self.corpora = corpora
        self.budget = budget_bytes
        self.levels = levels
        self.max_batch = max_batch
        self.gpj = GPJSON(device)          # batches (this thread)
        self._load_gpj = GPJSON(device)    # loads and releases (loader thread)
        self.resident: collections.OrderedDict[str, File] = collections.OrderedDict()
        self.loading: set[str] = set()
        self.used = 0
        self.loads = 0
        self.evictions = 0
        self._cv = threading.Condition()
        self._jobs: queue.Queue = queue.Queue()
        self._error: BaseException | None = None
        self._loader = threading.Thread(target=self._loader_loop, name="gpjson-loader", daemon=True)
        self._loader.start()
        # one batch for the server's life: its page-locked result buffer is
        # allocated once and reused by every iteration
        self._batch = self.gpj.batch()

    # -- loader thread -------------------------------------------------------
    def _loader_loop(self) -> None:
        while True:
            job = self._jobs.get()
            if job is None:
                return
            kind, name, f = job
            try:
                if kind == "release":
                    f.release()
                    continue
                f = self._load_gpj.load_bytes_indexed(self.corpora[name], self.levels)
                with self._cv:
                    self.resident[name] = f
                    self.loading.discard(name)
                    self.loads += 1
                    self._cv.notify_all()
            except BaseException as e:  # surfaced by serve()
                with self._cv:
                    self._error = e
                    self.loading.discard(name)
                    self._cv.notify_all()

    # -- admission ------------------------------------------------------------
    def _admit(self, name: str, needed: set[str]) -> bool:
        """True when `name` is resident; otherwise starts its load (after
        evicting least recently used corpora not in `needed`)."""
        with self._cv:
            if name in self.resident:
                self.resident.move_to_end(name)
                return True
            if name in self.loading:
                return False
            cost = resident_bytes(self.corpora[name].size, self.levels)
            while self.used + cost > self.budget:
                victim = next((v for v in self.resident if v not in needed), None)
                if victim is None:
                    if not self.resident and not self.loading:
                        raise MemoryError(f"corpus {name} ({cost} B resident) exceeds the {self.budget} B budget")
                    return False  # wait for room
                f = self.resident.pop(victim)
                self.used -= resident_bytes(self.corpora[victim].size, self.levels)
                self.evictions += 1
                self._jobs.put(("release", victim, f))
            self.used += cost
            self.loading.add(name)
        self._jobs.put(("load", name, None))
        return False

    def preload(self, names) -> None:
        for name in names:
            self._admit(name, set(names))
        with self._cv:
            while any(n in self.loading for n in names):
                if self._error:
                    raise self._error
                self._cv.wait(0.05)

    # -- serving -------------------------------------------------------------
    def serve(self, requests: list[Request], per_request: bool = False, keep_results: bool = False) -> ServeStats:
        """Runs `requests` (ascending arrival) in real time; per_request=True
        runs each request alone (the baseline form)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        batch = self._batch
        pending: collections.deque[Request] = collections.deque()
        nxt, finished, batches = 0, 0, 0
        t0 = time.perf_counter()
        try:
            while finished < len(reqs):
                if self._error:
                    raise self._error
                now = time.perf_counter() - t0
                while nxt < len(reqs) and reqs[nxt].arrival <= now:
                    pending.append(reqs[nxt])
                    nxt += 1
                needed = {r.corpus for r in pending}
                ready = [r for r in pending if self._admit(r.corpus, needed)]
                if not ready:
                    wait = reqs[nxt].arrival - now if nxt < len(reqs) else 0.05
                    with self._cv:
                        self._cv.wait(max(0.0, min(wait, 0.05)))
                    continue
                take = ready[:1] if per_request else ready[: self.max_batch]
                batch.clear()
                items = []
                for r in take:
                    with self._cv:
                        f = self.resident[r.corpus]
                    items.append(batch.add(f, r.paths))
                batch.run()
                batches += 1
                done = time.perf_counter() - t0
                taken = set(map(id, take))
                for r, it in zip(take, items):
                    r.done = done
                    if keep_results:
                        r.result = batch.result(it)
                pending = collections.deque(r for r in pending if id(r) not in taken)
                finished += len(take)
        finally:
            batch.clear()
        last = max(r.done for r in reqs) if reqs else 0.0
        first = min(r.arrival for r in reqs) if reqs else 0.0
        return ServeStats(
            requests=len(reqs), seconds=last - first,
            latencies_ms=[1000.0 * (r.done - r.arrival) for r in reqs],
            batches=batches, loads=self.loads, evictions=self.evictions,
        )

    def close(self) -> None:
        with self._cv:
            files = list(self.resident.values())
            self.resident.clear()
        for f in files:
            self._jobs.put(("release", "", f))
        self._jobs.put(None)
        self._loader.join(timeout=60)
        self._batch.release()
        self.gpj.close()
        self._load_gpj.close()


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
