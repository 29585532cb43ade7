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
