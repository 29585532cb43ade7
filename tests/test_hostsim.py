"""The device code's arithmetic (word_ops.cuh, interp.cuh) compiled for the
host and run in the index kernel's tile/word decomposition, against the
oracle.  Catches logic errors without a GPU; the same sources are compiled
for sm_100a into the product library."""

from __future__ import annotations

import ctypes
import random

import numpy as np
import pytest

from gpjson_b200 import datagen
from oracle import oracle
from tests.conftest import fixture_bytes
from tests.test_gpu_index import FIXTURE_NAMES, adversarial_bytes


def hs_index(hostsim, data: bytes, levels: int):
    f = np.frombuffer(data, dtype=np.uint8)
    n = f.size
    words = (n + 63) // 64
    nl = np.zeros(n + 1, np.int64)
    st = np.zeros(max(words, 1), np.uint64)
    lv = np.zeros(max(words * levels, 1), np.uint64)
    cnt = hostsim.hs_build_index(f.ctypes.data, n, levels, st.ctypes.data, lv.ctypes.data, nl.ctypes.data, n + 1)
    return nl[:cnt], st[:words], lv[: words * levels].reshape(levels, words)


def hs_index_lines(hostsim, data: bytes, levels: int):
    f = np.frombuffer(data, dtype=np.uint8)
    n = f.size
    words = (n + 63) // 64
    nl = np.zeros(n + 1, np.int64)
    st = np.full(max(words, 1), 0xDEAD, np.uint64)
    lv = np.full(max(words * levels, 1), 0xDEAD, np.uint64)
    cnt = hostsim.hs_build_index_lines(f.ctypes.data, n, levels, st.ctypes.data, lv.ctypes.data, nl.ctypes.data,
                                       n + 1)
    if cnt < 0:
        return None
    return nl[:cnt], st[:words], lv[: words * levels].reshape(levels, words)


def check_index(hostsim, data: bytes, levels: int, expect_regular=None):
    want = oracle.Index(data, levels)
    nl, st, lv = hs_index(hostsim, data, levels)
    assert np.array_equal(nl, want.newlines)
    assert np.array_equal(st, want.strings)
    assert np.array_equal(lv, want.levels)
    lines = hs_index_lines(hostsim, data, levels)
    if expect_regular is not None:
        assert (lines is not None) == expect_regular
    if lines is not None:  # the line-parallel result, when accepted, is exact
        assert np.array_equal(lines[0], want.newlines)
        assert np.array_equal(lines[1], want.strings)
        assert np.array_equal(lines[2], want.levels)


def test_escape_mask_random_words(hostsim):
    rng = random.Random(7)
    for it in range(20000):
        bs = rng.getrandbits(64) | (rng.getrandbits(64) if it % 2 else 0)
        if it % 97 == 0:
            bs = (1 << 64) - 1
        cin = rng.getrandbits(1)
        cout = ctypes.c_uint32()
        got = hostsim.hs_escaped_mask(bs, cin, ctypes.byref(cout))
        e, want = cin, 0
        for i in range(64):
            if e:
                want |= 1 << i
            e = (1 - e) if (bs >> i) & 1 else 0
        keep = ~bs & ((1 << 64) - 1)  # exact on every byte that is not a backslash
        assert (got & keep) == (want & keep)
        assert cout.value == e


@pytest.mark.parametrize("rel", FIXTURE_NAMES)
def test_fixtures(hostsim, rel):
    check_index(hostsim, fixture_bytes(rel), 16)


@pytest.mark.parametrize("seed", range(12))
def test_random_structured_bytes(hostsim, seed):
    rng = random.Random(seed)
    alphabet = b'{}[]:,"\\\n ab' if seed % 2 else b'\\\\\\"\n{}[]:,a '
    for n in [0, 1, 63, 64, 65, 16383, 16384, 16385, 50000]:
        data = bytes(rng.choice(alphabet) for _ in range(n))
        check_index(hostsim, data, rng.choice([1, 3, 16]))


def test_tile_straddling_escapes(hostsim):
    # backslash runs ending exactly at, before and after 16 KiB tile starts
    for run in range(1, 9):
        for shift in range(-3, 4):
            pre = b"a" * (16384 - run + shift)
            data = pre + b"\\" * run + b'"x"{"k":[1,2]}\n' + b"y" * 100
            check_index(hostsim, data, 3)


def test_generated(hostsim):
    check_index(hostsim, datagen.tweets(1 << 20).tobytes(), 4, expect_regular=True)
    check_index(hostsim, adversarial_bytes(3 << 20), 16, expect_regular=True)


def test_line_parallel_rejects_irregular(hostsim):
    good = datagen.tweets(200000).tobytes()
    cut = good.index(b"\n", 100000)
    for bad in [b'{"a": "x\ny"}', b'{"a": [1, 2}', b'{"a": 1}}', b'"open']:
        data = good[:cut] + b"\n" + bad + good[cut:]
        check_index(hostsim, data, 4, expect_regular=False)
    # brackets and quotes balanced inside a line are fine, whatever the bytes
    check_index(hostsim, good[:cut] + b'\n{"s":"\\\\\\"\\\\","t":[{}]}' + good[cut:], 4, expect_regular=True)


def colon_bitmap(f: np.ndarray, strings: np.ndarray) -> np.ndarray:
    """':' bytes outside strings, one bit per byte (the fused kernel's colon mask)."""
    words = strings.size
    in_str = np.unpackbits(strings.view(np.uint8), bitorder="little")[: f.size].astype(bool)
    bits = np.zeros(words * 64, dtype=np.uint8)
    bits[: f.size] = (f == ord(":")) & ~in_str
    return np.packbits(bits, bitorder="little").view(np.uint64).copy()


def test_interpreter_matches_oracle(hostsim):
    rng = random.Random(3)
    base = [
        fixture_bytes("query_gpu_function/simple_single_line.ldjson"),
        b'{"a": {"b": "a"},"b": {"a": "c" }}',
        b'{"a":[1,[2,3],{"b":4}],"c":{"d":[]}}',
        b'{"a" :[ {"b":[0,1,{"c":"x"}]} , 7 ], "d": "\\"a\\":1"}',
        b'  {"k\\"ey": 1, "key": [ ], "x":{"y":[[],[1]]}}  ',
        b'{"a":' + b" " * 100 + b'1, "b": [' + b" " * 70 + b'2]}',
        b'{"a": \n' + b" " * 90 + b'1}',  # a value's whitespace runs on into the next line
        # deep enough for every size of the interpreter's register state
        b'{"p":{"q":[[{"r":{"s":[0,{"t":{"u":[1,2,{"v":{"w":"deep"}}]}}]}}]]}}',
        # a key check that starts before the key's own string (at the
        # previous string's closing quote) and one at an escaped quote
        b'{"cd","ab":1, "e\\"lang":2, "lang":3}',
    ]
    paths = [
        "$.user.lang", "$.user.values[2]", "$.user.values[0:3]", "$.a.a", "$.a[1][0]", "$.a[2].b",
        "$.c.d[0]", "$.c.d[0:2]", "$.user.lang[?(@ == 'nl')]", "$[0]", "$.b.a", "$.a[0].b[2].c",
        "$.key[0]", "$.x.y[1][0]", "$.x.y[0:2]", "$['k\\\"ey']", "$.d", "$.a", "$.b[0]",
        "$.p.q[0][0].r.s[1].t.u[2].v.w", "$.p.q[0][0].r.s[0:2]", "$.p.q[0][0].r.s[1].t.u[0:3]",
        "$[',\"ab']", "$.lang", "$['\"lang']",
    ]
    for trial in range(40):
        lines = [rng.choice(base) for _ in range(rng.randint(1, 20))]
        lines.append(bytes(rng.choice(b'{}[]:,"\\ ab') for _ in range(rng.randint(0, 80))))
        rng.shuffle(lines)
        data = b"\n".join(lines)
        for path in paths:
            ir, depth, slots = oracle.compile_path(path)
            idx = oracle.Index(data, depth)
            want = oracle.find_value(data, idx.newlines, idx.strings, idx.levels, depth, ir, slots)
            f = np.frombuffer(data, dtype=np.uint8)
            irb = np.frombuffer(ir, dtype=np.uint8)
            ptrs = (ctypes.c_void_p * 1)(irb.ctypes.data)
            colon = colon_bitmap(f, idx.strings)
            # plain, with the fused kernel's colon jumps, with its packed level
            # state, and with the 32-bit interpreter's 64-bit fallbacks forced
            for colon_ptr, packed in ((None, 0), (colon.ctypes.data, 0), (colon.ctypes.data, 1), (None, 2),
                                      (colon.ctypes.data, 3), (colon.ctypes.data, 4)):
                got = np.empty_like(want)
                hostsim.hs_find_values(f.ctypes.data, f.size, idx.newlines.ctypes.data, len(idx.newlines),
                                       idx.strings.ctypes.data, idx.levels.ctypes.data, 1, ptrs, slots,
                                       got.ctypes.data, colon_ptr, packed)
                assert np.array_equal(got, want), (path, data[:120], colon_ptr is not None, packed)


@pytest.mark.parametrize("lines", [0, 1, 31, 32, 33, 1000])
@pytest.mark.parametrize("nq", [1, 3, 4, 17])
@pytest.mark.parametrize("stride", [256, 768, 1792, 227328])
def test_query_item_numbering(hostsim, lines, nq, stride):
    """Every (line, query) pair of a file is one item of the find_value
    kernels, whatever the grid stride and the file's offset in a batch; the
    32 lanes of a warp share one query on 32 consecutive lines."""
    for item_begin in (0, 96, 4128):
        pairs = np.full((max(1, lines * nq), 2), -7, dtype=np.int64)
        count = hostsim.hs_query_items(item_begin, lines, nq, stride, pairs.ctypes.data)
        assert count == lines * nq
        got = pairs[:count]
        want = {(i, q) for i in range(lines) for q in range(nq)}
        assert set(map(tuple, got.tolist())) == want
        # items in numbering order: warps of 32 share the query, lines consecutive
        full = np.full(((lines + 31) // 32 * 32 * nq, 2), -1, dtype=np.int64)
        k = 0
        for blk in range((lines + 31) // 32):
            for w in range(nq):
                n_real = min(32, lines - 32 * blk)
                full[k:k + n_real] = got[:n_real]
                got = got[n_real:]
                k += 32
        for w0 in range(0, len(full), 32):
            warp = full[w0:w0 + 32]
            real = warp[warp[:, 0] >= 0]
            assert len(set(real[:, 1].tolist())) <= 1
            assert (np.diff(real[:, 0]) == 1).all()


def test_classification_every_byte_value(hostsim):
    """The SWAR byte classes of the index kernels are exact for all 256 byte
    values at every position of a word (each value once at each of the 64
    positions, among the other values)."""
    rng = np.random.default_rng(11)
    words = []
    for pos in range(64):
        for v in range(256):
            w = rng.integers(0, 256, 64, dtype=np.uint8)
            w[pos] = v
            words.append(w)
    data = np.concatenate(words)
    out = np.zeros(len(words) * 7, dtype=np.uint64)
    hostsim.hs_classify(data.ctypes.data, len(words), out.ctypes.data)
    got = out.reshape(-1, 7)
    b = data.reshape(-1, 64)
    classes = [b == ord("\\"), b == ord('"'), b == ord("\n"), (b == ord("{")) | (b == ord("[")),
               (b == ord("}")) | (b == ord("]")),
               np.isin(b, np.frombuffer(b"{}[]:,", dtype=np.uint8)), b == ord(":")]
    weights = (np.uint64(1) << np.arange(64, dtype=np.uint64))
    for k, flags in enumerate(classes):
        want = (flags.astype(np.uint64) * weights).sum(axis=1, dtype=np.uint64)
        assert np.array_equal(got[:, k], want), k


def test_index_union_slots_equal_single_indices(hostsim):
    """A union path `...[i,j,k]...` (the PATH_INDEX_UNIONS extension) gives
    in slot b what the path with the single index of branch b gives, line by
    line, under the device interpreter (compiled here, checked against the
    oracle's evaluation of the single-index paths).  Unions compile like the
    reference's ranges, so an index step after one behaves as after a range
    in the reference (the inner array's element counter carries over from
    one branch to the next: only the first branch finds its element); those
    paths are checked against the equivalent range instead."""
    import gpjson_b200 as gj

    rng = random.Random(17)
    docs = [
        b'{"a":[{"b":0},{"b":1},{"b":2},{"b":[3]},{"c":4}],"x":{"y":[[1,2],[3],[],[4,[5,6]]]}}',
        b'{"a":[ 10 , {"b":"q"} ,[1,{"b":2}], "s" ],"x":{"y":[]}}',
        b'{"a":[],"x":{"y":[[0],[1],[2],[3]]}}',
        b'{"a":{"b":1},"x":[1,2,3]}',
        b'  {"x":{"y":[[ ], [ 7 , 8 , 9 ] , [{"z":1}] ]}, "a":[{"b":{"c":[1,2,3]}},{}]}',
    ]
    unions = {
        "$.a[0,2,3].b": ["$.a[0].b", "$.a[2].b", "$.a[3].b"],
        "$.a[1,4]": ["$.a[1]", "$.a[4]"],
        "$.x.y[0,3]": ["$.x.y[0]", "$.x.y[3]"],
        # an index step after the union: as after the range over the same indices
        "$.x.y[1,2][0,1]": ["$.x.y[1:3][0:2]"],
    }
    for _ in range(20):
        lines = [rng.choice(docs) for _ in range(rng.randint(1, 12))]
        data = b"\n".join(lines)
        f = np.frombuffer(data, dtype=np.uint8)
        for union, singles in unions.items():
            c = gj.compile_path(union, gj.PATH_INDEX_UNIONS)
            idx = oracle.Index(data, c.max_depth)
            irb = np.frombuffer(c.bytecode, dtype=np.uint8)
            ptrs = (ctypes.c_void_p * 1)(irb.ctypes.data)
            got = np.empty((1, len(idx.newlines), c.num_results, 2), dtype=np.int64)
            hostsim.hs_find_values(f.ctypes.data, f.size, idx.newlines.ctypes.data, len(idx.newlines),
                                   idx.strings.ctypes.data, idx.levels.ctypes.data, 1, ptrs, c.num_results,
                                   got.ctypes.data, None, 0)
            if len(singles) == 1:  # the equivalent range: all slots
                ir, depth, slots = oracle.compile_path(singles[0])
                sidx = oracle.Index(data, depth)
                want = oracle.find_value(data, sidx.newlines, sidx.strings, sidx.levels, depth, ir, slots)
                assert np.array_equal(got[0], want), (union, data[:80])
                continue
            assert c.num_results == len(singles)
            for b, single in enumerate(singles):
                ir, depth, slots = oracle.compile_path(single)
                sidx = oracle.Index(data, depth)
                want = oracle.find_value(data, sidx.newlines, sidx.strings, sidx.levels, depth, ir, slots)
                assert np.array_equal(got[0, :, b], want[:, 0]), (union, single, data[:80])


@pytest.mark.parametrize("threads", [1, 3, 16])
def test_slice_reader_reads_ranges(hostsim, tmp_path, threads):
    """gpj::SliceReader (gpj_file_open's reader): ranges of every size,
    including ragged ones shorter than a slice per thread, read back to back
    through one reader equal the file's bytes; a range past the end of the
    file fails (the file shrank) and reading stops there."""
    rng = np.random.default_rng(5)
    data = rng.integers(0, 256, size=(5 << 20) + 4321, dtype=np.uint8)
    path = tmp_path / "f.bin"
    data.tofile(path)
    spans = [(0, 1), (7, 3 << 20), (0, data.size), (data.size - 17, 17), ((1 << 20) + 5, 999), (123, 0)]
    pos = np.array([p for p, _ in spans], dtype=np.int64)
    ln = np.array([n for _, n in spans], dtype=np.int64)
    out = np.zeros(int(ln.sum()), dtype=np.uint8)
    got = hostsim.hs_read_ranges(str(path).encode(), out.ctypes.data, pos.ctypes.data, ln.ctypes.data, len(spans),
                                 threads)
    assert got == len(spans)
    want = np.concatenate([data[p:p + n] for p, n in spans])
    assert np.array_equal(out, want)
    # a short read ends the sequence at that range
    pos2 = np.array([0, data.size - 10, 0], dtype=np.int64)
    ln2 = np.array([100, 20, 100], dtype=np.int64)
    out2 = np.zeros(220, dtype=np.uint8)
    assert hostsim.hs_read_ranges(str(path).encode(), out2.ctypes.data, pos2.ctypes.data, ln2.ctypes.data, 3,
                                  threads) == 1
    assert hostsim.hs_read_ranges(str(tmp_path / "missing").encode(), out2.ctypes.data, pos2.ctypes.data,
                                  ln2.ctypes.data, 1, threads) == -1


def test_result_buffers_keep_the_largest(hostsim):
    """gpj::ResultBuffers (host memory of gpj_result): a released buffer is
    handed to the next result that fits in it, the larger of two released
    buffers is the one kept (up to 512 MiB), and a new buffer starts zeroed
    (touched before the copy into it)."""
    import ctypes

    b = hostsim.hs_rb_new()
    try:
        cap = ctypes.c_uint64()
        p1 = hostsim.hs_rb_take(b, 1000, ctypes.byref(cap))
        assert p1 and cap.value == 1000
        assert np.ctypeslib.as_array((ctypes.c_int64 * 1000).from_address(p1)).sum() == 0
        hostsim.hs_rb_give(b, p1, cap.value)
        p2 = hostsim.hs_rb_take(b, 600, ctypes.byref(cap))
        assert p2 == p1 and cap.value == 1000  # reused, with its full capacity
        p3 = hostsim.hs_rb_take(b, 2000, ctypes.byref(cap))
        assert p3 != p1 and cap.value == 2000  # nothing kept: a new buffer
        hostsim.hs_rb_give(b, p2, 1000)
        hostsim.hs_rb_give(b, p3, 2000)  # the larger one is kept
        p4 = hostsim.hs_rb_take(b, 1500, ctypes.byref(cap))
        assert p4 == p3 and cap.value == 2000
        p5 = hostsim.hs_rb_take(b, 3000, ctypes.byref(cap))  # larger than the kept one
        assert p5 != p4 and cap.value == 3000
        hostsim.hs_rb_give(b, p5, cap.value)
        hostsim.hs_rb_give(b, p4, 2000)  # smaller than the kept one: freed
        p6 = hostsim.hs_rb_take(b, 2500, ctypes.byref(cap))
        assert p6 == p5 and cap.value == 3000
        hostsim.hs_rb_give(b, p6, cap.value)
        assert hostsim.hs_rb_keep_elems() == 64 << 20  # 512 MiB at most are kept
    finally:
        hostsim.hs_rb_delete(b)
