"""Benchmark: input GB/s of the index + fused-query pass on one NDJSON file.

Workload (default): the 2 GiB tweet-like NDJSON file, one index build
(4 levels) and the four queries $.user.lang, $.id, $.user.followers_count,
$.entities.hashtags[0].text evaluated fused in one pass.  A step is one
index + query pass over the whole file with the input resident in HBM
(`value`), or through the C ABI with pinned host input and host results
(`e2e`: H2D of the file, index, query, D2H of the offsets).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (launched by torch.distributed.run) every rank processes its own
file of the same shape (weak scaling, no data-path collective); times are
the max over ranks.  `--impl reference` times the reference algorithm's CPU
implementation (the oracle restatement of Sequential.java, multi-threaded)
on a bounded sample of the same workload on this host's cores.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

QUERIES = ["$.user.lang", "$.id", "$.user.followers_count", "$.entities.hashtags[0].text"]
FILE_BYTES = 1 << 31
LEVELS = 4
PROFILE_TRAFFIC = ROOT / "profiles" / "dram_traffic_index_kernels_256MiB.json"


class Workload:
    """One NDJSON file of a configuration's shape and its queries."""

    def __init__(self, name: str, nbytes: int, levels: int, queries: list[str], kind: str, seed: int):
        self.name, self.bytes, self.levels, self.queries, self.kind, self.seed = name, nbytes, levels, queries, kind, seed

    def generate(self, n: int, rank: int = 0, out=None):
        from gpjson_b200 import datagen

        if self.kind == "tweets":
            return datagen.tweets(n, seed=self.seed + rank, p_empty_hashtags=0.3, out=out)
        return datagen.adversarial(n, seed=self.seed + rank, out=out)

    def describe(self, n: int, lines: int) -> str:
        what = ("tweet-like NDJSON" if self.kind == "tweets" else
                "adversarial NDJSON (lines 100 B-1 MiB log-uniform, nesting 1-16, arrays of 0-1000 numbers, "
                "backslash runs)")
        return (f"{what}, {n} B per GPU ({lines} lines), one index build ({self.levels} levels) + "
                f"{len(self.queries)} queries fused in one pass over it")


# the 2 GiB tweet-like file with its four queries (the headline), and the
# 4 GiB adversarial file with its three queries
TWEETS = Workload("tweets", FILE_BYTES, LEVELS, QUERIES, "tweets", 0x67706A73 + 1)
ADVERSARIAL = Workload("adversarial", 4 << 30, 5, ["$.a.b.c.d", "$.arr[5]", "$.x[0].y[2].z"], "adversarial",
                       0x67706A73 + 2)


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--bytes", type=int, default=None,
                    help="input file size (default: 2 GiB tweet-like, 4 GiB adversarial)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample", type=int, default=512 << 20, help="bytes of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", choices=["default", "fused", "index"], default="default",
                    help="default: gpj_index_query_device as shipped (index kernel, then one find_value "
                         "launch for all queries); fused: the queries evaluated inside the index kernel; "
                         "index: index only (diagnostic)")
    ap.add_argument("--workload", choices=["tweets", "adversarial", "batched", "serving"], default="tweets",
                    help="tweets: the 2 GiB single-file headline; adversarial: the 4 GiB adversarial file with "
                         "its three queries; batched: 512 files of 4 KiB-64 MiB, 1-8 "
                         "queries each, one batch vs per-file calls; serving: 64 resident corpora, Poisson "
                         "requests, continuous batching vs per-request")
    ap.add_argument("--requests", type=int, default=20000, help="serving: number of requests")
    ap.add_argument("--no-tune", action="store_true", help="keep the library's default launch shapes")
    ap.add_argument("--chunk-tiles", type=int, default=None,
                    help="after tuning: index and query the resident file in chunks of this many 30 KiB tiles "
                         "(a multiple of 1024; 0 = whole-file passes)")
    ap.add_argument("--no-extras", action="store_true",
                    help="default run: skip the adversarial, batched and serving measurements added to its line")
    ap.add_argument("--rate", type=float, default=2000.0, help="serving: arrivals per second")
    return ap.parse_args(argv)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Max of a per-rank scalar (times are reported as the slowest rank)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gbs(world: int, bytes_per_rank: int, ms_per_step: float) -> float:
    """Input GB/s of the whole job: every rank indexes its own file of
    bytes_per_rank bytes per step; the step time is the slowest rank's."""
    return world * bytes_per_rank / (ms_per_step / 1000) / 1e9


def barrier(world: int, device=None) -> None:
    if world > 1:
        import torch.distributed as dist

        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"],
                stdout=self.file, stderr=subprocess.DEVNULL,
            )
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.25)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "", 1).isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": reasons,
            "samples": len(rows),
        }


def measured_peak_gbs() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic(key: str):
    """DRAM bytes of one launch of an index kernel (`key`) and the input
    bytes it processed, from the committed ncu summary
    (profiles/dram_traffic_index_kernels_256MiB.json); the caller scales them
    to its input size."""
    if not PROFILE_TRAFFIC.exists():
        return None
    try:
        entry = json.loads(PROFILE_TRAFFIC.read_text())[key]
        return entry
    except Exception:
        return None


def cpu_baseline(data_np, n_sample: int, threads_all: bool, w: Workload = TWEETS):
    """The oracle port of the reference's sequential path on a sample."""
    from oracle import oracle

    sample = data_np[:n_sample]
    # cut at a line boundary so the sample is whole lines
    cut = int(n_sample)
    while cut > 0 and sample[cut - 1] != 10:
        cut -= 1
    sample = sample[:cut]
    t0 = time.perf_counter()
    idx = oracle.Index(sample, w.levels, mt=threads_all)
    oracle.query(sample, w.queries, mt=threads_all, index=idx)
    dt = time.perf_counter() - t0
    return cut / dt / 1e9, cut, dt, (oracle.num_threads() if threads_all else 1)


def run_reference(args, rank: int, world: int) -> None:
    """CPU reference arm: the oracle restatement of Sequential on all host
    threads, over the same whole file as our arm (same generator, seed, size
    and queries)."""
    if rank != 0:
        return
    from oracle import oracle

    w = ADVERSARIAL if args.workload == "adversarial" else TWEETS
    n = args.bytes or w.bytes
    data = w.generate(n)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        idx = oracle.Index(data, w.levels, mt=True)
        oracle.query(data, w.queries, mt=True, index=idx)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    ms = 1000 * statistics.mean(times)
    value = n / (ms / 1000) / 1e9
    cores = oracle.num_threads()
    lines = len(idx.newlines)
    line = {
        "impl": "reference",
        "metric": "input GB/s (index+query)",
        "value": round(value, 4),
        "unit": "GB/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": {
            "workload": w.describe(n, lines),
            "queries": w.queries,
            "bytes_per_gpu": n,
            "lines_per_gpu": lines,
        },
        "cpu_baseline": {
            "value": round(value, 4),
            "unit": "GB/s",
            "cores": cores,
            "kind": "port",
            "sample": f"the whole {n} B file of the GPU arm's workload, index ({w.levels} levels) + "
                      f"{len(w.queries)} queries per step",
        },
        "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local: int) -> None:
    import torch

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)
    w = ADVERSARIAL if args.workload == "adversarial" else TWEETS
    result = measure_file(args, w, rank, world, local, device)
    if rank == 0 and world == 1 and w is TWEETS and not args.no_extras and args.bytes is None:
        # the other configurations on the same GPU in the same run, bounded
        # so the default run stays within minutes
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup, sub.e2e_steps = min(args.steps, 5), 3, 1
        sub.cpu_sample = 128 << 20
        adv = measure_file(sub, ADVERSARIAL, rank, world, local, device)
        result["adversarial"] = {k: adv[k] for k in ("value", "ms_per_step", "config", "kernels_ms", "roofline",
                                                     "e2e", "cpu_baseline") if k in adv}
        sub.steps, sub.warmup = min(args.steps, 3), 1
        bat = measure_batched(sub)
        result["batched"] = {k: bat[k] for k in ("metric", "value", "unit", "ms_per_step", "config", "input_gbs",
                                                 "per_file_calls", "batched_vs_per_file", "resident_replay")}
        sub.requests = min(args.requests, 4000)
        srv = measure_serving(sub)
        result["serving"] = {k: srv[k] for k in ("metric", "value", "unit", "config", "latency_ms", "live",
                                                 "cold_start", "saturated_batched", "saturated_per_request",
                                                 "batched_vs_per_request_qps")}
        result["batched_vs_per_file"] = bat["batched_vs_per_file"]
        result["batched_vs_per_request_qps"] = srv["batched_vs_per_request_qps"]
        result["served_p50_ms"] = srv["latency_ms"]["p50"]
        result["served_p99_ms"] = srv["latency_ms"]["p99"]
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def measure_file(args, w: Workload, rank: int, world: int, local: int, device) -> dict:
    """The single-file workload `w`: device-resident passes (value), the end
    to end passes through the C ABI (e2e), the roofline of the index kernel
    and the CPU baseline; returns the JSON line's fields."""
    import ctypes

    import numpy as np
    import torch

    import gpjson_b200 as gj

    QUERIES, LEVELS = w.queries, w.levels
    n = args.bytes or w.bytes
    host = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    host_np = host.numpy()
    w.generate(n, rank, out=host_np)
    dev = host.to(device, non_blocking=False)
    torch.cuda.synchronize()

    g = gj.GPJSON(local)
    # one explicit stream carries our kernels and the timing events
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)
    g.set_stream(stream.cuda_stream)
    lib, ctx = g._native.lib, g._native.h
    compiled = [gj.compile_path(q) for q in QUERIES]
    bufs = [ctypes.create_string_buffer(c.bytecode, len(c.bytecode)) for c in compiled]
    ptrs = (ctypes.c_void_p * len(compiled))(*[ctypes.addressof(b) for b in bufs])
    lens = (ctypes.c_size_t * len(compiled))(*[len(c.bytecode) for c in compiled])
    slots = max(c.num_results for c in compiled)
    # launch shapes chosen by the autotuner on a 256 MiB sample of the same file
    tuned = None
    if not args.no_tune:
        from gpjson_b200 import tune

        cut = min(n, 256 << 20)
        while cut > 1 and host_np[cut - 1] != 10:
            cut -= 1
        tuned = tune.tune(g, dev[:cut], QUERIES, LEVELS, device=local, persist=False, workload=w.name)
    if args.chunk_tiles is not None:
        g.set_tuning(chunk_tiles=args.chunk_tiles)
    f = g.from_device(dev.data_ptr(), n, keepalive=dev)

    # first pass sizes the index and result buffers
    f.build_index(LEVELS)
    lines = f.num_lines
    out = torch.empty((len(QUERIES), lines, slots, 2), dtype=torch.int64, device=device)

    g.set_query_fusion(args.mode == "fused")

    def step(ev=None):
        """One pass: index + the queries in one pass over it, input in HBM."""
        if ev:
            ev[0].record(stream)
        if args.mode == "index":
            g._native.check(lib.gpj_index_build(ctx, f._h, LEVELS))
        else:
            g._native.check(lib.gpj_index_query_device(ctx, f._h, LEVELS, len(compiled), ptrs, lens, slots,
                                                       out.data_ptr(), lines))
        if ev:
            ev[1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    launches0 = g.kernel_launches()
    exact0 = g.timings()["exact_index_fallbacks"]
    lib.gpj_reset_timings(ctx)
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world, device)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(args.steps):
        step(evs[k])
    end.record(stream)
    torch.cuda.synchronize()
    barrier(world, device)
    clock_info = clocks.stop()
    launches = g.kernel_launches() - launches0
    exact_builds = g.timings()["exact_index_fallbacks"] - exact0
    # per-kernel device times: the library brackets each kernel phase with
    # CUDA events on this same stream (gpj_get_timings)
    phase_ms: dict[str, list[float]] = {}
    for ph in g.timings()["phases"]:
        phase_ms.setdefault(ph["name"], []).append(ph["device_ms"])
    kernel_ms = {k: statistics.mean(v) for k, v in phase_ms.items()}
    total_ms = start.elapsed_time(end)
    pass_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    total_ms = max_over_ranks(total_ms, world, device)
    ms_per_step = total_ms / args.steps
    value = whole_job_gbs(world, n, ms_per_step)

    # correctness spot check of the timed output against one solo pass
    if args.mode != "index":
        g.set_query_fusion(False)
        solo = f.run(compiled)
        assert np.array_equal(solo, out.cpu().numpy()), "device results differ from a solo pass"

    # ---- end to end through the C ABI with host buffers ----------------------
    res_host = torch.empty((len(QUERIES), lines, slots, 2), dtype=torch.int64, pin_memory=True)
    # one call: copy, index and queries pipelined (gpj_file_from_host_query);
    # beside it the two-call form (gpj_file_from_host_indexed, then gpj_query)
    e2e_times, e2e_two_call = [], []
    e2e_lines = ctypes.c_int64()
    for k in range(1 + args.e2e_steps):
        for form in ("two", "one"):  # the one-call form last: its results are checked below
            barrier(world, device)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            h = ctypes.c_void_p()
            if form == "one":
                g._native.check(lib.gpj_file_from_host_query(ctx, host.data_ptr(), n, LEVELS, len(compiled), ptrs,
                                                             lens, slots, res_host.data_ptr(), res_host.numel(),
                                                             ctypes.byref(e2e_lines), ctypes.byref(h)))
            else:
                g._native.check(lib.gpj_file_from_host_indexed(ctx, host.data_ptr(), n, LEVELS, ctypes.byref(h)))
                g._native.check(lib.gpj_query(ctx, h, len(compiled), ptrs, lens, slots, res_host.data_ptr(),
                                              res_host.numel()))
            lib.gpj_file_release(h)
            dt = time.perf_counter() - t0
            if k > 0:
                (e2e_times if form == "one" else e2e_two_call).append(dt)
    e2e_s = max_over_ranks(statistics.mean(e2e_times), world, device)
    e2e_two_s = max_over_ranks(statistics.mean(e2e_two_call), world, device)
    # the e2e ceiling: a plain pinned host-to-device copy of the same bytes
    scratch = torch.empty(n, dtype=torch.uint8, device=device)
    scratch.copy_(host, non_blocking=True)
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    scratch.copy_(host, non_blocking=True)
    c1.record(stream)
    torch.cuda.synchronize()
    h2d_gbs = n / (c0.elapsed_time(c1) / 1000) / 1e9
    del scratch
    if args.mode != "index":
        assert np.array_equal(res_host.numpy(), out.cpu().numpy()), "e2e results differ"
    e2e_value = world * n / e2e_s / 1e9

    # ---- value extraction (gpj_query_values): the matched values gathered on
    # the device into one compact buffer instead of the (start, end) pairs
    value_info = None
    if args.mode != "index":
        lib.gpj_reset_timings(ctx)
        vals = f.query_values(QUERIES)
        vphase = {ph["name"]: ph["device_ms"] for ph in g.timings()["phases"]}
        value_info = {
            "gather_and_copy_ms": round(vphase.get("gather_values", float("nan")), 4),
            "values": int((vals.kinds == gj.VALUE_PRESENT).sum()),
            "value_bytes": len(vals.data),
            "pair_bytes": int(out.numel() * 8),
            "note": "gpj_query_values on the resident index: device time of the gather (sizes, scan, byte copy) "
                    "and of the copies of kinds + offsets + value bytes to pageable host memory",
        }
        del vals

    # ---- roofline of the dominant kernel ----------------------------------------
    # Algorithmic bytes of one index (+query) pass = the input bytes n (each
    # byte is read once; the index it writes is reported beside it).  The
    # dominant kernel is the index kernel (phase "build_index": the
    # standalone tile kernel and the newline index kernels, or
    # "index_and_query" when the queries run inside the line kernel).
    peak, peak_kind = measured_peak_gbs()
    words = (n + 63) // 64
    # string index, leveled bitmaps, the ':' bitmap and the newline index
    index_bytes = 8 * words * (2 + LEVELS) + 8 * lines
    dom = "index_and_query" if "index_and_query" in kernel_ms else "build_index"
    dom_ms = kernel_ms[dom]
    achieved = n / (dom_ms / 1000) / 1e9
    # which kernel the timed builds ran: the exact kernel for input the line
    # kernels refuse, else the standalone tile kernel (or the line kernel with
    # the queries, or the chunked pass's kernels)
    if exact_builds > 0:
        dom_kernel = "index_kernel (exact, decoupled look-back; the line kernels refuse this input)"
    elif dom == "build_index":
        dom_kernel = "tile_index_kernel (+ the two newline index kernels)"
    elif args.mode == "fused":
        dom_kernel = "line_index_kernel (with the queries)"
    else:
        dom_kernel = "chunked pass: tile_index_kernel, newline index and find_value per chunk"
    traffic = None
    # the committed captures: the standalone tile kernel's build of tweets,
    # the exact kernel's build of the adversarial file
    t = ncu_traffic("exact_index_kernel" if exact_builds > 0 else "index_kernel")
    if dom == "build_index" and t and t.get("bytes") and t.get("input_bytes"):
        traffic = round(t["bytes"] * n / t["input_bytes"])

    result = {
        "metric": "input GB/s (index+query)",
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": {
            "workload": w.describe(n, lines),
            "mode": args.mode,
            "queries": QUERIES,
            "bytes_per_gpu": n,
            "lines_per_gpu": lines,
            "l2": (f"input larger than L2 ({n / 2**20:.0f} MiB vs 126 MB)" if n > 126_000_000
                   else f"input within L2 ({n / 2**20:.0f} MiB vs 126 MB): not a valid bench size"),
            "parallelism": f"replicas x{world} (one file per GPU)",
        },
        "pass_ms": round(pass_ms, 4),
        "kernels_ms": {k: round(v, 4) for k, v in kernel_ms.items()},
        "roofline": {
            "bound": "hbm",
            "kernel": dom_kernel,
            "achieved": round(achieved, 1),
            "peak": peak,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "traffic": traffic,
            "algorithmic_bytes": n,
            "index_bytes_written": index_bytes,
            "peak_kind": f"{peak_kind} copy bandwidth",
        },
        "step_frac_of_hbm": round(value / world / peak, 4),
        "e2e": {
            "value": round(e2e_value, 3),
            "unit": "GB/s",
            "h2d_bytes_per_step": n,
            "d2h_bytes_per_step": int(res_host.numel() * 8),
            "path": "gpj_file_from_host_query: copy overlapped with indexing and with each chunk's queries, "
                    "results to pinned host",
            "two_call_gbs": round(world * n / e2e_two_s / 1e9, 3),
            "two_call_path": "gpj_file_from_host_indexed (copy overlapped with indexing) + gpj_query",
            "pinned_h2d_copy_gbs": round(h2d_gbs, 2),
        },
        "value_extraction": value_info,
        "tuning": (None if tuned is None else
                   {"chosen": tuned["tuning"], "applied": g.tuning(),
                    "search": "gpjson_b200.tune coordinate search on a 256 MiB sample of the same file "
                              "(index build + query pass per setting, CUDA-event device ms)",
                    "candidates_ms": tuned["measured_ms"]}),
        "gpu_launches": int(launches),
        "clocks": clock_info,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cut, dt, cores = cpu_baseline(host_np, min(args.cpu_sample, n), threads_all=False, w=w)
        result["cpu_baseline"] = {
            "value": round(v, 4),
            "unit": "GB/s",
            "cores": cores,
            "kind": "port",
            "sample": f"{cut} B prefix (whole lines) of the same file, index + {len(QUERIES)} queries, {dt:.1f} s",
        }
    f.release()
    g.close()
    del dev, out, host
    torch.cuda.empty_cache()
    return result


def batched_corpus(seed: int = 0x67706A73 + 3, files: int = 512):
    """512 file sizes, lognormal clipped to 4 KiB-64 MiB (about 6 GiB in all),
    three in four from the tweet-like generator, the rest adversarial; 1-8
    queries per file from the 32-path pool."""
    import numpy as np

    from gpjson_b200 import serve

    rng = np.random.default_rng(seed)
    sizes = np.clip(rng.lognormal(mean=15.6, sigma=1.4, size=files), 4 << 10, 64 << 20).astype(np.int64)
    kinds = rng.random(files) < 0.75
    paths = [[serve.PATH_POOL[i] for i in rng.choice(32, size=int(rng.integers(1, 9)), replace=False)]
             for _ in range(files)]
    return sizes, kinds, paths


def run_batched(args) -> None:
    print(json.dumps(measure_batched(args)), flush=True)


def measure_batched(args) -> dict:
    """Batched workload: every step indexes all 512 files and evaluates their
    queries, once as one gpj_batch_run, once as 512 gpj_query_paths calls."""
    import torch

    import gpjson_b200 as gj
    from gpjson_b200 import datagen

    sizes, kinds, paths = batched_corpus()
    total = int(sizes.sum())
    dev = []
    for i, (n, tweet) in enumerate(zip(sizes, kinds)):
        seed = datagen.SEED_BASE + 1000 + i
        host = datagen.tweets(int(n), seed=seed) if tweet else datagen.adversarial(int(n), seed=seed)
        dev.append(torch.from_numpy(host).to("cuda"))
    torch.cuda.synchronize()
    g = gj.GPJSON(0)
    nq = sum(len(p) for p in paths)

    def fresh_files():  # unindexed views of the resident inputs
        return [g.from_device(t.data_ptr(), t.numel(), keepalive=t) for t in dev]

    b = g.batch()  # reused: its page-locked result buffer is allocated once

    def batched_step():
        fs = fresh_files()
        b.clear()
        for f, p in zip(fs, paths):
            b.add(f, p)
        t0 = time.perf_counter()
        b.run()
        dt = time.perf_counter() - t0
        b.clear()
        for f in fs:
            f.release()
        return dt

    def per_file_step():
        fs = fresh_files()
        t0 = time.perf_counter()
        for f, p in zip(fs, paths):
            f.query_paths(p)
        dt = time.perf_counter() - t0
        for f in fs:
            f.release()
        return dt

    for _ in range(args.warmup):
        batched_step()
        per_file_step()
    tb = [batched_step() for _ in range(args.steps)]
    tp = [per_file_step() for _ in range(max(1, min(args.steps, 3)))]
    mb, mp = statistics.mean(tb), statistics.mean(tp)
    # the same requests again on the resident indexes: after two runs the
    # batch's query phase is a CUDA graph, replayed by every later run
    res_files = fresh_files()
    rb = g.batch()
    for f, p in zip(res_files, paths):
        rb.add(f, p)
    for _ in range(3):
        rb.run()
    g._native.lib.gpj_reset_timings(g._native.h)
    tr = []
    for _ in range(max(3, args.steps)):
        t0 = time.perf_counter()
        rb.run()
        tr.append(time.perf_counter() - t0)
    replayed = sum(1 for ph in g.timings()["phases"] if ph["name"] == "batch_query_replay")
    rb.release()
    for f in res_files:
        f.release()
    mr = statistics.mean(tr)
    line = {
        "metric": "queries/s (batched index+query)",
        "value": round(nq / mb, 1),
        "unit": "queries/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1000 * mb, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": {"workload": f"{len(sizes)} NDJSON files of 4 KiB-64 MiB ({total} B), 3/4 tweet-like, 1/4 "
                               f"adversarial; {nq} queries, 1-8 per file from a 32-path pool; each step indexes "
                               "every file and evaluates its queries, results copied to the host",
                   "files": len(sizes), "bytes": total, "queries": nq},
        "input_gbs": round(total / mb / 1e9, 2),
        "per_file_calls": {"ms_per_step": round(1000 * mp, 3), "queries_per_s": round(nq / mp, 1),
                           "input_gbs": round(total / mp / 1e9, 2)},
        "batched_vs_per_file": round(mp / mb, 2),
        "resident_replay": {"ms_per_step": round(1000 * mr, 3), "queries_per_s": round(nq / mr, 1),
                            "graph_replays": replayed, "runs": len(tr),
                            "note": "the same batch run again on the resident indexes: its query phase (find_value, "
                                    "long-line warps, result copy) replayed as one CUDA graph"},
    }
    b.release()
    g.close()
    del dev
    torch.cuda.empty_cache()
    return line


def run_serving(args) -> None:
    print(json.dumps(measure_serving(args)), flush=True)


def measure_serving(args) -> dict:
    """Serving workload: 64 corpora of 1 MiB-1 GiB (log-uniform), requests
    arriving Poisson with Zipf(1.1) corpus popularity, a 120 GiB budget;
    continuous batching, then the per-request form on a saturated sample."""
    import numpy as np

    from gpjson_b200 import datagen, serve

    rng = np.random.default_rng(0x67706A73 + 4)
    sizes = np.exp(rng.uniform(np.log(1 << 20), np.log(1 << 30), size=64)).astype(np.int64)
    corpora = {}
    for i, n in enumerate(sizes):
        seed = datagen.SEED_BASE + 2000 + i
        corpora[f"c{i:02d}"] = datagen.tweets(int(n), seed=seed) if i % 4 else datagen.adversarial(int(n), seed=seed)
    names = list(corpora)
    total = int(sizes.sum())
    srv = serve.Server(corpora, budget_bytes=120 << 30)
    try:
        # cold: corpora load when first requested; then the same arrival
        # process again with every corpus resident (steady state)
        cold = srv.serve(serve.poisson_requests(names, args.requests, rate=args.rate, seed=21)).summary()
        reqs = serve.poisson_requests(names, args.requests, rate=args.rate)
        live = srv.serve(reqs).summary()
        # saturated: every request available at once; each form runs once
        # untimed first (result buffers grown, all corpora resident)
        sample = serve.poisson_requests(names, 2000, rate=1e9, seed=11)
        srv.serve([serve.Request(0.0, r.corpus, list(r.paths)) for r in sample])
        batched = srv.serve(sample).summary()
        solo_sample = [serve.Request(0.0, r.corpus, list(r.paths)) for r in sample[:500]]
        srv.serve([serve.Request(0.0, r.corpus, list(r.paths)) for r in solo_sample], per_request=True)
        solo = srv.serve(solo_sample, per_request=True).summary()
    finally:
        srv.close()
    line = {
        "metric": "served queries/s (p50/p99 latency)",
        "value": live["queries_per_s"],
        "unit": "queries/s",
        "n_gpus": 1,
        "steps": 1,
        "warmup": 0,
        "ms_per_step": round(1000 * live["seconds"], 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": {"workload": f"64 corpora of 1 MiB-1 GiB log-uniform ({total} B), {args.requests} requests "
                               f"Poisson at {args.rate:.0f}/s, Zipf 1.1 popularity, 1 path each from a 32-path "
                               "pool, 120 GiB resident budget, continuous batching (at most 512 requests per "
                               "batch); value and latency with the corpora resident",
                   "corpora": 64, "bytes": total},
        "latency_ms": {"p50": live["p50_ms"], "p99": live["p99_ms"], "mean": live["mean_ms"]},
        "live": live,
        "cold_start": cold,
        "saturated_batched": batched,
        "saturated_per_request": solo,
        "batched_vs_per_request_qps": round(batched["queries_per_s"] / max(solo["queries_per_s"], 1e-9), 2),
    }
    return line


def main(argv=None) -> None:
    args = parse_args(argv)
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "batched":
        if rank == 0:
            run_batched(args)
        return
    if args.workload == "serving":
        if rank == 0:
            run_serving(args)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
