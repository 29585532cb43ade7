"""GPU parity of gpj_build_index_device_noalloc (the index build that uses a
static __device__ scratch array instead of allocating) against
gpj_build_index_device on the same device buffers, two calls in a row, on
well-formed NDJSON (line-parallel kernel) and on pretty-printed JSON (exact
kernel fallback).  The file name keeps it last in collection so it also runs
after every other GPU test has used the device."""

from __future__ import annotations

import ctypes
import json
import random

import numpy as np
import pytest

from gpjson_b200 import _lib, datagen
from oracle import oracle


def pretty_json(seed: int, records: int) -> bytes:
    rng = random.Random(seed)

    def value(depth):
        r = rng.random()
        if depth > 5 or r < 0.3:
            return rng.choice([rng.randint(-9999, 9999), "s\\\"q" * rng.randint(0, 3), None, True, 1.5])
        if r < 0.65:
            return {f"k{i}": value(depth + 1) for i in range(rng.randint(0, 4))}
        return [value(depth + 1) for _ in range(rng.randint(0, 4))]

    return json.dumps([value(0) for _ in range(records)], indent=2).encode()


def device_buffers(torch, n: int, levels: int):
    words = (n + 63) // 64
    # filled with a pattern so a word either entry point leaves unwritten shows up
    d_str = torch.full((words,), -1, dtype=torch.int64, device="cuda")
    d_lvl = torch.full((levels * words,), -1, dtype=torch.int64, device="cuda")
    d_nl = torch.full((n // 16 + 16,), -1, dtype=torch.int64, device="cuda")
    return d_str, d_lvl, d_nl


def build(gpjson, torch, d_file, n: int, levels: int, noalloc: bool):
    lib = gpjson._native.lib
    d_str, d_lvl, d_nl = device_buffers(torch, n, levels)
    lines = ctypes.c_int64(-1)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    if noalloc:
        rc = lib.gpj_build_index_device_noalloc(
            ctypes.c_void_p(stream), d_file.data_ptr(), n, levels, d_str.data_ptr(), d_lvl.data_ptr(),
            d_nl.data_ptr(), d_nl.numel(), ctypes.byref(lines),
        )
        assert rc == 0, f"gpj_build_index_device_noalloc returned {rc}"
    else:
        rc = lib.gpj_build_index_device(
            gpjson._native.h, d_file.data_ptr(), n, levels, d_str.data_ptr(), d_lvl.data_ptr(), d_nl.data_ptr(),
            d_nl.numel(), ctypes.byref(lines),
        )
        gpjson._native.check(rc)
    torch.cuda.synchronize()
    return (lines.value, d_nl[: lines.value].cpu().numpy(), d_str.cpu().numpy(), d_lvl.cpu().numpy())


def assert_same(a, b):
    assert a[0] == b[0], "line count"
    assert np.array_equal(a[1], b[1]), "newline index"
    assert np.array_equal(a[2], b[2]), "string index"
    assert np.array_equal(a[3], b[3]), "leveled bitmaps"


@pytest.mark.gpu
@pytest.mark.parametrize(
    "kind,levels",
    [("ndjson", 4), ("ndjson", 16), ("pretty", 16)],
)
def test_noalloc_matches_context_entry(gpjson, kind, levels):
    import torch

    data = datagen.tweets(8 << 20).tobytes() if kind == "ndjson" else pretty_json(7, 3000)
    n = len(data)
    d_file = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
    before = gpjson.timings()["exact_index_fallbacks"]
    want = build(gpjson, torch, d_file, n, levels, noalloc=False)
    # the pretty input is one the line-parallel kernel flags: the context
    # entry needed the exact kernel, so the no-alloc entry's equal result
    # shows that its own fallback ran
    fallbacks = gpjson.timings()["exact_index_fallbacks"] - before
    assert (fallbacks >= 1) if kind == "pretty" else (fallbacks == 0)
    first = build(gpjson, torch, d_file, n, levels, noalloc=True)
    second = build(gpjson, torch, d_file, n, levels, noalloc=True)
    assert_same(first, want)
    assert_same(second, want)
    ref = oracle.Index(data, levels)
    assert np.array_equal(first[1], ref.newlines)
    assert np.array_equal(first[2].view(np.uint64), ref.strings)


@pytest.mark.gpu
def test_noalloc_alternates_inputs(gpjson):
    """Back-to-back calls on different inputs: the scratch array (tile
    states, counter, status) carries nothing from one call to the next."""
    import torch

    a = datagen.tweets(4 << 20).tobytes()
    b = pretty_json(11, 1500)
    da = torch.frombuffer(bytearray(a), dtype=torch.uint8).cuda()
    db = torch.frombuffer(bytearray(b), dtype=torch.uint8).cuda()
    want_a = build(gpjson, torch, da, len(a), 8, noalloc=False)
    want_b = build(gpjson, torch, db, len(b), 8, noalloc=False)
    for _ in range(2):
        assert_same(build(gpjson, torch, da, len(a), 8, noalloc=True), want_a)
        assert_same(build(gpjson, torch, db, len(b), 8, noalloc=True), want_b)


@pytest.mark.gpu
def test_noalloc_epoch_wrap(gpjson):
    """The tile states in the static scratch carry the launch's 16-bit epoch
    and are cleared when it wraps.  2 x 65,536 + 16 builds alternate two
    multi-tile inputs, so every epoch value is used again after the wrap by
    the other input (the cycle of 65,535 values is odd): a tile state left
    from before the wrap would be taken for the current launch's and shift
    the other input's newline offsets.  Every build must equal its input's
    build through the context entry."""
    import torch

    lib = gpjson._native.lib
    inputs = []
    for seed, size in ((41, 192 << 10), (42, 160 << 10)):
        data = datagen.tweets(size, seed=datagen.SEED_BASE + seed).tobytes()
        d_file = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
        want = build(gpjson, torch, d_file, len(data), 4, noalloc=False)
        d_str, d_lvl, d_nl = device_buffers(torch, len(data), 4)
        inputs.append((d_file, len(data), want[0], torch.from_numpy(want[1]).cuda(), d_str, d_lvl, d_nl))
    assert inputs[0][2] != inputs[1][2]
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    lines = ctypes.c_int64(-1)
    for k in range(2 * 65536 + 16):
        d_file, n, want_lines, want_nl, d_str, d_lvl, d_nl = inputs[k & 1]
        rc = lib.gpj_build_index_device_noalloc(
            ctypes.c_void_p(stream), d_file.data_ptr(), n, 4, d_str.data_ptr(), d_lvl.data_ptr(), d_nl.data_ptr(),
            d_nl.numel(), ctypes.byref(lines),
        )
        assert rc == 0, (k, rc)
        assert lines.value == want_lines, k
        assert torch.equal(d_nl[:want_lines], want_nl), k


@pytest.mark.gpu
def test_noalloc_rejects_oversized_input(gpjson):
    """Inputs above the scratch array's limit are refused before any launch
    (the pointer is never read: the size check comes first)."""
    import torch

    lib = gpjson._native.lib
    d = torch.zeros(1024, dtype=torch.int64, device="cuda")
    lines = ctypes.c_int64(-1)
    n = (256 << 20) + 64
    rc = lib.gpj_build_index_device_noalloc(
        None, d.data_ptr(), n, 4, d.data_ptr(), d.data_ptr(), d.data_ptr(), d.numel(), ctypes.byref(lines)
    )
    assert rc == _lib.GPJ_ELIMIT
    assert lines.value == -1
    rc = lib.gpj_build_index_device_noalloc(
        None, d.data_ptr(), 4096, 17, d.data_ptr(), d.data_ptr(), d.data_ptr(), d.numel(), ctypes.byref(lines)
    )
    assert rc == _lib.GPJ_ELIMIT


@pytest.mark.gpu
def test_noalloc_refuses_a_capturing_stream(gpjson):
    """A call on a stream that is being captured into a graph is refused
    (GPJ_EINVAL) before it touches the stream: every call reads its status
    back and waits for its stream, which capture does not allow."""
    import torch

    lib = gpjson._native.lib
    data = datagen.tweets(1 << 20, seed=datagen.SEED_BASE + 31).tobytes()
    n = len(data)
    d_file = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
    d_str, d_lvl, d_nl = device_buffers(torch, n, 4)
    lines = ctypes.c_int64(-1)
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph, stream=side):
        rc = lib.gpj_build_index_device_noalloc(
            ctypes.c_void_p(side.cuda_stream), d_file.data_ptr(), n, 4, d_str.data_ptr(), d_lvl.data_ptr(),
            d_nl.data_ptr(), d_nl.numel(), ctypes.byref(lines),
        )
        d_str.add_(0)  # some captured work
    assert rc == _lib.GPJ_EINVAL and lines.value == -1
    torch.cuda.synchronize()
