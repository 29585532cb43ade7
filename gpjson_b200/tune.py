"""Autotuner for the launch shapes of gpj_tuning (gpj_set_tuning).

The reference's launch shapes are fixed (8x1024 threads for its index
kernels, 512x1024 for find_value: stages/CombinedIndex.java:28-56,
functions/QueryFunction.java:201-241).  Here the resident CTAs per SM of
the standalone index kernel and of find_value, and the line length above
which find_value gives a line a whole warp, are searched on a sample of the
caller's workload: one knob at a time, each candidate timed with the
library's CUDA-event phase times of one gpj_index_query_device pass (index
build + queries; whole-file or chunk by chunk, the fourth knob), the best
kept.  Results do not depend on these shapes, only speed does.

The choice is stored per device (name and SM count) in a JSON file under
$GPJSON_TUNING_DIR (default ~/.cache/gpjson_b200) and applied by
`apply()`; the environment variables GPJSON_LONG_LINE_BYTES,
GPJSON_QUERY_CTAS_PER_SM, GPJSON_INDEX_CTAS_PER_SM and GPJSON_CHUNK_TILES
override it.
"""

from __future__ import annotations

import json
import os
import statistics
from collections.abc import Callable
from pathlib import Path

KNOBS = ("index_ctas_per_sm", "query_ctas_per_sm", "long_line_bytes", "chunk_tiles")
ENV = {"long_line_bytes": "GPJSON_LONG_LINE_BYTES", "query_ctas_per_sm": "GPJSON_QUERY_CTAS_PER_SM",
       "index_ctas_per_sm": "GPJSON_INDEX_CTAS_PER_SM", "chunk_tiles": "GPJSON_CHUNK_TILES"}
# candidates per knob (0 = the library's default: the occupancy maximum, 64 KiB,
# or whole-file passes)
CANDIDATES = {
    "index_ctas_per_sm": [0, 2, 3, 4],
    "query_ctas_per_sm": [0, 2, 4, 6],
    "long_line_bytes": [0, 16384, 262144, -1],
    "chunk_tiles": [0, 2048],
}


def search(measure: Callable[[dict], float], start: dict | None = None,
           candidates: dict[str, list[int]] | None = None, rounds: int = 2) -> tuple[dict, dict]:
    """Coordinate descent: for each knob in turn, every candidate with the
    others at their current best; `rounds` sweeps.  `measure(setting)`
    returns a time (lower is better).  Returns (best setting, the time of
    every setting measured, keyed by its JSON)."""
    cand = candidates or CANDIDATES
    best = dict(start or {k: 0 for k in KNOBS})
    seen: dict[str, float] = {}

    def timed(setting: dict) -> float:
        key = json.dumps(setting, sort_keys=True)
        if key not in seen:
            seen[key] = float(measure(dict(setting)))
        return seen[key]

    best_t = timed(best)
    for _ in range(rounds):
        changed = False
        for knob in cand:
            for v in cand[knob]:
                trial = dict(best, **{knob: v})
                t = timed(trial)
                if t < best_t:
                    best, best_t, changed = trial, t, True
        if not changed:
            break
    return best, seen


def device_key(name: str, sms: int) -> str:
    return "".join(c if c.isalnum() else "_" for c in f"{name}_{sms}sm")


def store_path(key: str) -> Path:
    root = Path(os.environ.get("GPJSON_TUNING_DIR", Path.home() / ".cache" / "gpjson_b200"))
    return root / f"tuning-{key}.json"


def save(key: str, setting: dict, measured: dict | None = None, workload: str = "") -> Path:
    p = store_path(key)
    p.parent.mkdir(parents=True, exist_ok=True)
    record = {"device": key, "tuning": {k: int(setting[k]) for k in KNOBS if k in setting}, "workload": workload,
              "measured_ms": measured or {}}
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(record, indent=1, sort_keys=True) + "\n")
    tmp.replace(p)
    return p


def load(key: str) -> dict:
    """The stored setting with the environment's overrides on top ({} when
    neither exists)."""
    out: dict = {}
    p = store_path(key)
    if p.exists():
        try:
            out.update(json.loads(p.read_text()).get("tuning", {}))
        except (OSError, ValueError):
            pass
    for knob, var in ENV.items():
        if os.environ.get(var, "").strip():
            out[knob] = int(os.environ[var])
    return out


def _device_key_of(device: int) -> str:
    import torch

    prop = torch.cuda.get_device_properties(device)
    return device_key(prop.name, prop.multi_processor_count)


def apply(gpjson, device: int = 0) -> dict:
    """Applies the stored / environment setting to a GPJSON context; returns
    what was applied."""
    setting = load(_device_key_of(device))
    if setting:
        gpjson.set_tuning(**{k: int(v) for k, v in setting.items() if k in KNOBS})
    return setting


def tune(gpjson, data, queries: list[str], levels: int, device: int = 0, repeats: int = 3, persist: bool = True,
         workload: str = "") -> dict:
    """Searches the launch shapes on `data` (a uint8 numpy array or torch
    CUDA tensor, a sample of the workload) with `queries`, applies the best
    to `gpjson` and (persist) stores it for the device.  Returns
    {"tuning": best, "measured_ms": {setting: ms}}."""
    import numpy as np
    import torch

    import gpjson_b200 as gj

    dev = data if isinstance(data, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(data)).to(
        torch.device("cuda", device))
    f = gpjson.from_device(dev.data_ptr(), dev.numel(), keepalive=dev)
    compiled = [gj.compile_path(q) for q in queries]
    lib, h = gpjson._native.lib, gpjson._native.h
    f.build_index(levels)
    slots = max(c.num_results for c in compiled)
    out = torch.empty((len(compiled), f.num_lines, slots, 2), dtype=torch.int64, device=dev.device)

    def measure(setting: dict) -> float:
        gpjson.set_tuning(**setting)
        f.index_and_query_device(compiled, levels, out.data_ptr(), f.num_lines, slots)  # warm
        lib.gpj_reset_timings(h)
        for _ in range(repeats):
            f.index_and_query_device(compiled, levels, out.data_ptr(), f.num_lines, slots)
        phases = gpjson.timings()["phases"]
        per = {}
        for ph in phases:
            per.setdefault(ph["name"], []).append(ph["device_ms"])
        # one pass = the sum of its phases (whole-file: index build + find_value)
        return sum(statistics.mean(v) for k, v in per.items()
                   if k in ("build_index", "find_value", "index_and_query"))

    try:
        best, seen = search(measure)
    finally:
        f.release()
    gpjson.set_tuning(**best)
    if persist:
        save(_device_key_of(device), best, seen, workload)
    return {"tuning": best, "measured_ms": {k: round(v, 4) for k, v in seen.items()}}
