"""GPU parity of the query path (index + fused find_value) against the
oracle: the reference's end-to-end known answers (QueryFunctionTest.java),
fused-versus-alone equality, generated NDJSON of the benchmark shapes and
random small documents with many path shapes."""

from __future__ import annotations

import random

import numpy as np
import pytest

import gpjson_b200 as gj
from gpjson_b200 import datagen
from oracle import oracle
from tests.conftest import FIXTURES, fixture_bytes
from tests.test_gpu_index import adversarial_bytes
from tests.test_oracle import KNOWN_ANSWERS, NOT_FOUND, SIMPLE

TWEET_PATHS = ["$.user.lang", "$.id", "$.user.followers_count", "$.entities.hashtags[0].text"]
ADV_PATHS = ["$.a.b.c.d", "$.arr[5]", "$.x[0].y[2].z"]


def flat_values(result: gj.Result) -> list:
    out = []
    for q in range(len(result)):
        arr = result[q]
        for line in range(len(arr)):
            out.extend(arr[line][k] for k in range(len(arr[line])))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("path,expected", KNOWN_ANSWERS, ids=[k[0] for k in KNOWN_ANSWERS])
def test_known_answers(gpjson, path, expected):
    result = gpjson.query(str(FIXTURES / SIMPLE), path)
    assert flat_values(result) == expected


@pytest.mark.gpu
def test_key_not_found_in_current_level(gpjson):
    result = gpjson.query(str(FIXTURES / NOT_FOUND), "$.a.a")
    assert all(v is None for v in flat_values(result))


@pytest.mark.gpu
def test_multiple_paths_one_call(gpjson):
    paths = [k[0] for k in KNOWN_ANSWERS]
    result = gpjson.query(str(FIXTURES / SIMPLE), paths)
    assert len(result) == len(paths)
    slots = max(len(k[1]) for k in KNOWN_ANSWERS)
    for q, (_, expected) in enumerate(KNOWN_ANSWERS):
        got = [result[q][0][k] for k in range(slots)]
        assert got == expected + [None] * (slots - len(expected))


def run_gpu(gpjson, data: bytes, paths: list[str]) -> np.ndarray:
    """Every device path: gpj_query_paths with the queries evaluated inside
    the index kernel and after it, and the separate index build + find_value
    call (gpj_query); they must agree."""
    compiled = [gj.compile_path(p) for p in paths]
    f = gpjson.load_bytes(data)
    try:
        two_pass = f.query_paths(paths)
        again = f.query_paths(paths)  # the resident index is reused: queries only
        f.build_index(max(c.max_depth for c in compiled))
        separate = f.run(compiled)
    finally:
        f.release()
    assert np.array_equal(again, two_pass), "query on the resident index differs"
    f = gpjson.load_bytes(data)  # a fresh file, so the index is built with the queries inside
    gpjson.set_query_fusion(True)
    try:
        fused = f.query_paths(paths)
    finally:
        gpjson.set_query_fusion(False)
        f.release()
    assert np.array_equal(fused, separate), "in-kernel and separate query paths differ"
    assert np.array_equal(two_pass, separate), "two-pass and separate query paths differ"
    return fused


@pytest.mark.gpu
def test_fused_equals_alone_and_oracle_tweets(gpjson):
    data = datagen.tweets(32 << 20).tobytes()
    fused = run_gpu(gpjson, data, TWEET_PATHS)
    want = oracle.query(data, TWEET_PATHS, mt=True)
    assert np.array_equal(fused, want)
    for q, p in enumerate(TWEET_PATHS):
        alone = run_gpu(gpjson, data, [p])
        assert np.array_equal(alone[0], fused[q]), p


@pytest.mark.gpu
def test_adversarial_against_oracle(gpjson):
    data = adversarial_bytes(48 << 20)
    got = run_gpu(gpjson, data, ADV_PATHS)
    want = oracle.query(data, ADV_PATHS, mt=True)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_random_documents_many_paths(gpjson):
    rng = random.Random(11)
    base = [
        fixture_bytes(SIMPLE),
        b'{"a": {"b": "a"},"b": {"a": "c" }}',
        b'{"a":[1,[2,3],{"b":4}],"c":{"d":[]}}',
        b'{"a" :[ {"b":[0,1,{"c":"x"}]} , 7 ], "d": "\\"a\\":1"}',
        b'  {"k\\"ey": 1, "key": [ ], "x":{"y":[[],[1]]}}  ',
    ]
    paths = [
        "$.user.lang", "$.user.values[2]", "$.user.values[0:3]", "$.a.a", "$.a[1][0]", "$.a[2].b",
        "$.c.d[0]", "$.c.d[0:2]", "$.user.lang[?(@ == 'nl')]", "$[0]", "$.b.a", "$.a[0].b[2].c",
        "$.key[0]", "$.x.y[1][0]", "$.x.y[0:2]", "$['k\\\"ey']", "$.d",
    ]
    lines = []
    for _ in range(20000):
        if rng.random() < 0.9:
            lines.append(rng.choice(base))
        else:
            lines.append(bytes(rng.choice(b'{}[]:,"\\ ab') for _ in range(rng.randint(0, 80))))
    data = b"\n".join(lines)
    got = run_gpu(gpjson, data, paths)
    want = oracle.query(data, paths)
    assert np.array_equal(got, want)


def random_documents(count: int, seed: int = 11) -> bytes:
    rng = random.Random(seed)
    base = [
        fixture_bytes(SIMPLE),
        b'{"a": {"b": "a"},"b": {"a": "c" }}',
        b'{"a":[1,[2,3],{"b":4}],"c":{"d":[]}}',
        b'{"a" :[ {"b":[0,1,{"c":"x"}]} , 7 ], "d": "\\"a\\":1"}',
        b'  {"k\\"ey": 1, "key": [ ], "x":{"y":[[],[1]]}}  ',
        b'{"a":' + b" " * 1500 + b'1, "b": [' + b" " * 700 + b'2]}',
    ]
    lines = []
    for _ in range(count):
        if rng.random() < 0.9:
            lines.append(rng.choice(base))
        else:
            lines.append(bytes(rng.choice(b'{}[]:,"\\ ab') for _ in range(rng.randint(0, 80))))
    return b"\n".join(lines)


@pytest.mark.gpu
def test_long_lines_on_a_warp_equal_oracle(gpjson):
    """Lines longer than the tuning's long_line_bytes are evaluated by a
    whole warp (the warp-wide bitmap searches and whitespace skips); with
    the threshold at 64 bytes almost every line takes that path (more than
    the hand-over list holds, so its overflow is evaluated per thread too),
    with -1 none does.  Results equal the oracle's either way, for the
    single-file and the batched launch."""
    paths = ["$.user.lang", "$.a[1][0]", "$.a[2].b", "$.c.d[0:2]", "$.user.lang[?(@ == 'nl')]", "$.b",
             "$.x.y[1][0]", "$['k\\\"ey']", "$.d", "$.a[0].b[2].c"]
    cases = [(random_documents(3000), paths), (adversarial_bytes(24 << 20), ADV_PATHS),
             (datagen.tweets(4 << 20, seed=datagen.SEED_BASE + 9).tobytes(), TWEET_PATHS)]
    try:
        for threshold in (64, -1, 0):
            gpjson.set_tuning(long_line_bytes=threshold)
            for data, ps in cases:
                want = oracle.query(data, ps, mt=True)
                f = gpjson.load_bytes(data)
                try:
                    assert np.array_equal(f.query_paths(ps), want), (threshold, ps)
                finally:
                    f.release()
            b = gpjson.batch()
            files = [gpjson.load_bytes(data) for data, _ in cases]
            try:
                items = [b.add(f, ps) for f, (_, ps) in zip(files, cases)]
                b.run()
                for it, (data, ps) in zip(items, cases):
                    want = oracle.query(data, ps, mt=True)
                    got = b.result(it)
                    assert np.array_equal(got[:, :, : want.shape[2]], want), (threshold, "batch", ps)
            finally:
                b.release()
                for f in files:
                    f.release()
    finally:
        gpjson.set_tuning(long_line_bytes=0)
    assert gpjson.tuning()["long_line_bytes"] == 65536


@pytest.mark.gpu
def test_empty_and_tiny_files(gpjson, tmp_path):
    for data in [b"", b"\n", b"{}", b'{"a":1}\n{"a":2}\n', b"\n\n\n"]:
        got = run_gpu(gpjson, data, ["$.a"])
        want = oracle.query(data, ["$.a"])
        assert np.array_equal(got, want), data


@pytest.mark.gpu
def test_index_zero_of_empty_array_quirk(gpjson, tmp_path):
    # [0] as the last step on [] stores (position of ']', -1) like find_value.cu;
    # reading that item fails like ResultItem.java (negative length).
    p = tmp_path / "q.ldjson"
    p.write_bytes(b'{"a": []}\n{"a": [5]}')
    result = gpjson.query(str(p), "$.a[0]")
    start, end = result[0][0].offsets(0)
    assert end == -1 and p.read_bytes()[start:start + 1] == b"]"
    with pytest.raises(gj.GPJSONException):
        result[0][0][0]
    assert result[0][1][0] == "5"


@pytest.mark.gpu
def test_fused_device_entry(gpjson):
    import torch

    data = datagen.tweets(12 << 20).tobytes()
    compiled = [gj.compile_path(p) for p in TWEET_PATHS]
    f = gpjson.load_bytes(data)
    try:
        f.build_index(4)
        lines = f.num_lines
        out = torch.full((len(compiled), lines, 1, 2), 7, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        want = oracle.query(data, TWEET_PATHS)
        for fusion in (False, True, False):
            gpjson.set_query_fusion(fusion)
            try:
                for _ in range(2):
                    out.fill_(7)
                    f.index_and_query_device(compiled, 4, out.data_ptr(), lines)
                    assert np.array_equal(out.cpu().numpy(), want), fusion
            finally:
                gpjson.set_query_fusion(False)
        small = torch.empty((len(compiled), lines - 1, 1, 2), dtype=torch.int64, device="cuda")
        with pytest.raises(gj.GPJSONException):
            f.index_and_query_device(compiled, 4, small.data_ptr(), lines - 1)
    finally:
        f.release()


@pytest.mark.gpu
def test_irregular_input_falls_back_exactly(gpjson):
    good = datagen.tweets(300000).tobytes()
    cut = good.index(b"\n", 150000)
    data = good[:cut] + b'\n{"user": {"lang": "x\ny"}}' + good[cut:]
    got = run_gpu(gpjson, data, TWEET_PATHS)
    assert np.array_equal(got, oracle.query(data, TWEET_PATHS))
    assert gpjson.timings()["exact_index_fallbacks"] >= 1


@pytest.mark.gpu
def test_errors(gpjson):
    path = str(FIXTURES / SIMPLE)
    with pytest.raises(gj.UnsupportedJSONPathException):
        gpjson.query(path, "$.a[*]")
    with pytest.raises(gj.JSONPathException):
        gpjson.query(path, "$.a b")
    with pytest.raises(gj.GPJSONException):
        gpjson.query(path, ["$.a"] * 256)
    with pytest.raises(gj.GPJSONException):
        gpjson.query(path, "$" + ".a" * 17)
    with pytest.raises(gj.GPJSONException):
        gpjson.query(str(FIXTURES / "does-not-exist.ldjson"), "$.a")


@pytest.mark.gpu
def test_file_open_reads_every_chunk(gpjson, tmp_path):
    """gpj_file_open reads 32 MiB chunks, each as slices read concurrently:
    a file of several chunks with a ragged tail holds the same bytes on the
    device as the input loaded from memory (the values of large members, the
    string and newline indexes, the query results); a directory fails like
    a missing file."""
    data = np.concatenate([datagen.tweets(100 << 20, seed=datagen.SEED_BASE + 77),
                           np.frombuffer(b'{"id": 7}', dtype=np.uint8)])
    path = tmp_path / "chunks.ldjson"
    data.tofile(path)
    f = gpjson.open(path)
    g = gpjson.load_bytes(data)
    try:
        assert f.size == data.size
        members = ["$.text", "$.user", "$.source", "$.entities"]
        got, want = f.query_values(members), g.query_values(members)
        assert got.data == want.data and np.array_equal(got.offsets, want.offsets)
        assert len(got.data) > data.size // 2
        assert np.array_equal(f.query_paths(TWEET_PATHS), g.query_paths(TWEET_PATHS))
        assert np.array_equal(f.string_index(), g.string_index())
        assert np.array_equal(f.newline_index(), g.newline_index())
    finally:
        f.release()
        g.release()
    with pytest.raises(gj.GPJSONException):
        gpjson.open(tmp_path)


@pytest.mark.gpu
def test_file_of_another_context(gpjson):
    """A file is used only with the context that made it: the query and
    index-read entry points refuse another context's file (GPJ_EINVAL)
    and leave it usable by its own."""
    other = gj.GPJSON(0)
    f = gpjson.load_bytes(b'{"a":1}\n{"a":[2]}\n')
    foreign = gj.File(other._native, f._h)  # the same handle through the other context
    try:
        f.build_index(2)
        q = [gj.compile_path("$.a")]
        with pytest.raises(gj.GPJSONException) as e:
            foreign.run(q)
        assert e.value.code == gj._lib.GPJ_EINVAL
        with pytest.raises(gj.GPJSONException):
            foreign.query_paths(["$.a"])
        with pytest.raises(gj.GPJSONException):
            foreign.newline_index()
        assert f.run(q)[0, :, 0, 0].tolist() == [5, 13, -1]
    finally:
        foreign._h = None  # the handle is f's to release
        f.release()
        other.close()


def _pipelined_case(case: str) -> tuple[np.ndarray, list[str]]:
    if case == "small":
        return datagen.tweets(1 << 20, seed=datagen.SEED_BASE + 61), TWEET_PATHS
    if case == "empty":
        return np.zeros(0, dtype=np.uint8), ["$.a"]
    if case == "many_lines":  # more lines than the newline index's first estimate
        return np.frombuffer(b'{"a":1}\n' * (15 << 20), dtype=np.uint8), ["$.a", "$.b"]
    base = datagen.tweets(150 << 20, seed=datagen.SEED_BASE + 62)
    if case == "ndjson":
        return base, TWEET_PATHS
    cut = int(np.flatnonzero(base[100 << 20:] == 10)[0]) + (100 << 20)
    extra = b'{"k":"' + b"x" * (70 << 20) + b'"}' if case == "long_line" else b'{"k": "a' + bytes([10]) + b'b"}'
    data = np.concatenate([base[: cut + 1], np.frombuffer(extra + b"\n", dtype=np.uint8), base[cut + 1:]])
    return data, TWEET_PATHS + ["$.k"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ndjson", "long_line", "raw_newline", "small", "empty", "many_lines"])
def test_pipelined_query_equals_load_then_query(gpjson, case):
    """gpj_file_from_host_query (each chunk's newline index and queries run
    while later chunks are still copied) equals the plain copy + index build
    + find_value call, including inputs that are indexed again after the
    copy (a line longer than a chunk, a raw newline in a string, more lines
    than the first estimate) and a result buffer that is too small."""
    data, paths = _pipelined_case(case)
    compiled = [gj.compile_path(p) for p in paths]
    levels = max(c.max_depth for c in compiled)
    f = gpjson.load_bytes(data)
    try:
        f.build_index(levels)
        want = f.run(compiled)
        lines = f.num_lines
    finally:
        f.release()
    out = np.full(want.size + 10, -5, dtype=np.int64)
    g, got = gpjson.load_bytes_query(data, levels, compiled, out=out)
    try:
        assert g.num_lines == lines
        assert np.array_equal(got, want)
        assert (out[want.size:] == -5).all()
    finally:
        g.release()
    if case in ("ndjson", "small"):
        g, got = gpjson.load_bytes_query(data, levels, compiled)  # no buffer: GPJ_ELIMIT, then gpj_query
        try:
            assert np.array_equal(got, want)
        finally:
            g.release()
    if case == "small":
        ref = oracle.query(data.tobytes(), paths)
        assert np.array_equal(want, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ndjson", "long_line", "raw_newline", "small", "many_lines"])
def test_chunked_resident_pass_equals_whole_file_pass(gpjson, case):
    """gpj_index_query_device with tuning.chunk_tiles (index kernel, newline
    index and find_value chunk by chunk over input already on the device)
    equals the whole-file pass, including inputs the chunks cannot index (a
    line longer than a chunk, a raw newline in a string: indexed again
    whole) and more lines than the first estimate; a too-small result
    buffer is refused."""
    import torch

    data, paths = _pipelined_case(case)
    compiled = [gj.compile_path(p) for p in paths]
    levels = max(c.max_depth for c in compiled)
    dev = torch.from_numpy(data).cuda()
    f = gpjson.from_device(dev.data_ptr(), dev.numel(), keepalive=dev)
    try:
        f.build_index(levels)
        want = f.run(compiled)
        lines = f.num_lines
        out = torch.full((len(compiled), lines, want.shape[2], 2), 7, dtype=torch.int64, device="cuda")
        for chunk in (1024, 2048):
            gpjson.set_tuning(chunk_tiles=chunk)
            try:
                for _ in range(2):
                    out.fill_(7)
                    f.index_and_query_device(compiled, levels, out.data_ptr(), lines)
                    assert f.num_lines == lines
                    assert np.array_equal(out.cpu().numpy(), want), (case, chunk)
                if lines > 1:
                    small = torch.empty((len(compiled), lines - 1, want.shape[2], 2), dtype=torch.int64,
                                        device="cuda")
                    with pytest.raises(gj.GPJSONException):
                        f.index_and_query_device(compiled, levels, small.data_ptr(), lines - 1)
            finally:
                gpjson.set_tuning(chunk_tiles=0)
        with pytest.raises(gj.GPJSONException):
            gpjson.set_tuning(chunk_tiles=1000)  # not a multiple of 1024
    finally:
        f.release()
    if case == "small":
        assert np.array_equal(want, oracle.query(data.tobytes(), paths))


@pytest.mark.gpu
def test_index_union_extension(gpjson):
    """`[i,j]` is rejected as the reference rejects it unless the context
    enables PATH_INDEX_UNIONS; then each index has its own result slot, equal
    to the single-index path's results (through query_paths and a batch)."""
    data = datagen.tweets(2 << 20, seed=datagen.SEED_BASE + 91).tobytes()
    union, singles = "$.entities.hashtags[0,2].text", ["$.entities.hashtags[0].text", "$.entities.hashtags[2].text"]
    f = gpjson.load_bytes(data)
    try:
        with pytest.raises(gj.UnsupportedJSONPathException):
            f.query_paths([union])
        gpjson.set_path_extensions(gj.PATH_INDEX_UNIONS)
        try:
            got = f.query_paths([union, "$.id"])
            b = gpjson.batch()
            try:
                it = b.add(f, [union])
                b.run()
                got_batch = b.result(it)
            finally:
                b.release()
        finally:
            gpjson.set_path_extensions(0)
        want = f.query_paths(singles)
    finally:
        f.release()
    assert got.shape[2] == 2
    for k in range(2):
        assert np.array_equal(got[0, :, k], want[k, :, 0])
        assert np.array_equal(got_batch[0, :, k], want[k, :, 0])
    assert (got[0, :, 1, 0] >= 0).sum() > 0 and (got[1, :, 1] == -1).all()
