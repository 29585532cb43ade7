"""Parity against the reference's own CUDA kernels, compiled from source
and driven with the reference's orchestration (oracle/_ref, built where the
reference sources are): on well-formed tweet-like NDJSON, the string index,
leveled bitmaps, newline index and every query's results of this library
equal the reference kernels' on the same GPU."""

from __future__ import annotations

import numpy as np
import pytest

import gpjson_b200 as gj
from gpjson_b200 import datagen
from oracle import ref_gpu

PATHS = ["$.user.lang", "$.id", "$.user.followers_count", "$.entities.hashtags[0].text"]


@pytest.mark.gpu
@pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref/libref_gpu.so not built (needs the reference sources)")
@pytest.mark.parametrize("size", [1 << 20, 24 << 20])
def test_equal_to_reference_kernels(gpjson, size):
    data = datagen.tweets(size, seed=datagen.SEED_BASE + 81, p_empty_hashtags=0.3)
    compiled = [gj.compile_path(p) for p in PATHS]
    levels = max(c.max_depth for c in compiled)
    slots = max(c.num_results for c in compiled)
    ref = ref_gpu.run(data, levels, [c.bytecode for c in compiled], slots, max_lines=size // 64 + 16)
    f = gpjson.load_bytes(data)
    try:
        f.build_index(levels)
        assert np.array_equal(f.newline_index(), ref["newlines"])
        assert np.array_equal(f.string_index(), ref["strings"])
        assert np.array_equal(f.leveled_bitmaps(levels), ref["levels"])
        got = f.run(compiled, slots)
    finally:
        f.release()
    assert np.array_equal(got, ref["results"])
    assert (got[:, :, 0, 0] >= 0).sum() > 0


def _compare_with_reference_kernels(gpjson, data: np.ndarray, paths: list[str]) -> np.ndarray:
    compiled = [gj.compile_path(p) for p in paths]
    levels = max(c.max_depth for c in compiled)
    slots = max(c.num_results for c in compiled)
    ref = ref_gpu.run(data, levels, [c.bytecode for c in compiled], slots, max_lines=data.size // 64 + 16)
    f = gpjson.load_bytes(data)
    try:
        f.build_index(levels)
        assert np.array_equal(f.newline_index(), ref["newlines"])
        assert np.array_equal(f.string_index(), ref["strings"])
        assert np.array_equal(f.leveled_bitmaps(levels), ref["levels"])
        got = f.run(compiled, slots)
    finally:
        f.release()
    assert np.array_equal(got, ref["results"])
    return got


@pytest.mark.gpu
@pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref/libref_gpu.so not built (needs the reference sources)")
def test_plain_small_configuration_equal_to_reference_kernels(gpjson):
    """64 MiB of tweet-like NDJSON from the generator's first seed, $.user.lang."""
    data = datagen.tweets(64 << 20, seed=datagen.SEED_BASE + 0, p_empty_hashtags=0.3)
    got = _compare_with_reference_kernels(gpjson, data, ["$.user.lang"])
    assert (got[0, :, 0, 0] >= 0).mean() > 0.99


@pytest.mark.gpu
@pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref/libref_gpu.so not built (needs the reference sources)")
def test_adversarial_sample_equal_to_reference_kernels(gpjson):
    """256 MiB of the adversarial generator (lines to 1 MiB, nesting to 16,
    backslash runs; well-formed, and index steps only meet arrays, so the
    reference kernels stay inside their buffers) with its three queries."""
    data = datagen.adversarial(256 << 20, seed=datagen.SEED_BASE + 2)
    got = _compare_with_reference_kernels(gpjson, data, ["$.a.b.c.d", "$.arr[5]", "$.x[0].y[2].z"])
    assert ((got[:, :, 0, 0] >= 0).sum(axis=1) > 0).all()


@pytest.mark.gpu
@pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref/libref_gpu.so not built (needs the reference sources)")
def test_faster_than_reference_kernels(gpjson, capsys):
    """The reference's GPU path (its kernels and host scans, input resident
    on the device, 4 queries each with a find_value launch) against this
    library's index build + one find_value launch, on the same 1 GiB of
    tweet-like NDJSON on the same GPU (the reference's counters overflow at
    2 GiB).  Prints both; requires a 20x margin."""
    import statistics

    size = 1 << 30
    data = datagen.tweets(size, seed=datagen.SEED_BASE + 1)
    compiled = [gj.compile_path(p) for p in PATHS]
    ref = ref_gpu.run(data, 4, [c.bytecode for c in compiled], 1, repeats=2, outputs=False)
    f = gpjson.load_bytes(data)
    try:
        for _ in range(2):
            f.build_index(4)
            f.run(compiled)
        gpjson._native.lib.gpj_reset_timings(gpjson._native.h)
        for _ in range(3):
            f.build_index(4)
            f.run(compiled)
        phases = {}
        for ph in gpjson.timings()["phases"]:
            phases.setdefault(ph["name"], []).append(ph["device_ms"])
    finally:
        f.release()
    ours_index = statistics.mean(phases["build_index"])
    ours_query = statistics.mean(phases["find_value"])
    ref_total = ref["index_ms"] + ref["query_ms"]
    ours_total = ours_index + ours_query
    with capsys.disabled():
        print(f"\n1 GiB, {ref['lines']} lines, 4 queries: reference kernels index {ref['index_ms']:.2f} ms + "
              f"queries {ref['query_ms']:.2f} ms = {size / ref_total / 1e6:.2f} GB/s; this library index "
              f"{ours_index:.3f} ms + queries {ours_query:.3f} ms = {size / ours_total / 1e6:.1f} GB/s; "
              f"{ref_total / ours_total:.0f}x")
    assert ours_total * 20 < ref_total
