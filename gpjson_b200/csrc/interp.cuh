// Per-line JSONPath bytecode interpreter over the leveled bitmaps.
//
// Semantics follow the reference interpreter find_value
// (gpjson/src/main/resources/com/koenv/gpjson/kernels/find_value.cu:21-263),
// which equals Sequential.findValue (sequential/Sequential.java:130-344).
// Instead of visiting every byte, the scan jumps from one structural bit of
// the current level to the next: bytes without such a bit cannot change the
// interpreter's state while it is searching (find_value.cu skips whole zero
// words for the same reason, :218-222).
//
// Where the reference reads out of bounds or trips a device assert, the
// behaviour below is fixed (marked [bounded]) and the test oracle implements
// the same choice.  __host__ __device__ so the test suite can run it on the
// CPU against the oracle.
#pragma once

#include <cstddef>
#include <cstdint>

#include "word_ops.cuh"

namespace gpj {

// One more than the deepest level a query may reach (16 key/index steps).
constexpr int kLevelSlots = 17;

struct LineView {
    const uint8_t* file;
    int64_t n;
    const uint64_t* string_index;
    const uint64_t* levels;  // [level][level_size]
    int64_t level_size;
    // Bytes at positions >= hi are not readable through this view (hi = n
    // for the whole file in device memory; a shared-memory view ends at the
    // last byte it holds).  A whitespace skip that reaches hi < n cannot be
    // finished here and the line is reported as deferred.
    int64_t hi;
    // Optional ':' outside strings, indexed like string_index.  When given,
    // a key search jumps only between structural colons and an index search
    // only between the other structural characters.
    const uint64_t* colon;
};

// kLineLong: run_line gave up on a whitespace skip longer than its skip
// bound (the caller evaluates the line again another way).
enum LineStatus : int { kLineDone = 0, kLineDeferred = 1, kLineLong = 2 };

GPJ_HD bool is_ws(uint8_t c) { return c == '\n' || c == '\r' || c == '\t' || c == ' '; }

// Every byte of x is one of the four whitespace bytes.
GPJ_HD bool all_ws32(uint32_t x) {
    return (eq_bytes(x, 0x20202020u) | eq_bytes(x, 0x0A0A0A0Au) | eq_bytes(x, 0x0D0D0D0Du) |
            eq_bytes(x, 0x09090909u)) == 0x80808080u;
}

// First position at or after j that is >= hi or not whitespace.  Short runs
// go byte by byte; a run longer than 32 bytes continues 32 aligned bytes per
// step (independent loads), so a skip over a long run of blanks does not
// wait for one memory round trip per byte.
template <typename P>
GPJ_HD P skip_ws(const uint8_t* file, P j, P hi) {
    for (int k = 0; k < 32; k++, ++j)
        if (j >= hi || !is_ws(file[j])) return j;
    for (; j < hi && (reinterpret_cast<uintptr_t>(file + j) & 7) != 0; ++j)
        if (!is_ws(file[j])) return j;
    for (; j + 32 <= hi; j += 32) {
        const uint32_t* w = reinterpret_cast<const uint32_t*>(file + j);
        uint32_t x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = w[i];
        bool all = true;
#pragma unroll
        for (int i = 0; i < 8; i++) all = all && all_ws32(x[i]);
        if (!all) break;
    }
    while (j < hi && is_ws(file[j])) ++j;
    return j;
}

// The bit helpers and the interpreter below are templates on the position
// type P: int64_t for positions in the file, int32_t for positions relative
// to a line's first word (run_line; half the integer work per step).

// First set bit of `bm` at a position in [from, limit), or `limit`.  After
// the first three words, four words are loaded per step (independent loads,
// so a long jump waits for a quarter of the dependent memory round trips);
// only words holding positions below `limit` are read.
template <typename P>
GPJ_HD P first_of4(P w, uint64_t a, uint64_t b, uint64_t c, uint64_t d, P limit) {
    P base = w;
    uint64_t x = a;
    if (!a) {
        base = b ? w + 1 : (c ? w + 2 : w + 3);
        x = b ? b : (c ? c : d);
    }
    const P p = (base << 6) + ctz64(x);
    return p < limit ? p : limit;
}

// `cw`/`cv`: a word of bm the caller already holds (index, value; cw = -1
// for none), used instead of reloading it; on return they hold the word the
// result was found in.
template <typename P>
GPJ_HD P next_bit(const uint64_t* bm, P from, P limit, P& cw, uint64_t& cv) {
    if (from >= limit) return limit;
    P w = from >> 6;
    const P wend = ((limit - 1) >> 6) + 1;
    const uint64_t first = w == cw ? cv : bm[w];
    const uint64_t m = first & (~0ull << (from & 63));
    if (m) {
        cw = w;
        cv = first;
        const P p = (w << 6) + ctz64(m);
        return p < limit ? p : limit;
    }
    // the next two words one at a time (most jumps end there), then four per step
    for (++w; w < wend && w < (from >> 6) + 3; ++w) {
        const uint64_t x = bm[w];
        if (x) {
            cw = w;
            cv = x;
            const P p = (w << 6) + ctz64(x);
            return p < limit ? p : limit;
        }
    }
    for (; w < wend; w += 4) {
        const uint64_t a = bm[w];
        const uint64_t b = w + 1 < wend ? bm[w + 1] : 0;
        const uint64_t c = w + 2 < wend ? bm[w + 2] : 0;
        const uint64_t d = w + 3 < wend ? bm[w + 3] : 0;
        if (a | b | c | d) {
            const P p = first_of4<P>(w, a, b, c, d, limit);
            cw = w + (a ? 0 : (b ? 1 : (c ? 2 : 3)));
            cv = a ? a : (b ? b : (c ? c : d));
            return p;
        }
    }
    return limit;
}

template <typename P>
GPJ_HD P next_bit(const uint64_t* bm, P from, P limit) {
    P cw = -1;
    uint64_t cv = 0;
    return next_bit<P>(bm, from, limit, cw, cv);
}

// First position in [from, limit) set in bm and (in `filt`, or not in it
// when `invert`), or `limit`; cw/cv as in next_bit, for the combined word
// bm[w] & (filt[w] ^ flip).
template <typename P>
GPJ_HD P next_bit_filtered(const uint64_t* bm, const uint64_t* filt, bool invert, P from, P limit, P& cw,
                           uint64_t& cv) {
    if (from >= limit) return limit;
    P w = from >> 6;
    const P wend = ((limit - 1) >> 6) + 1;
    const uint64_t flip = invert ? ~0ull : 0ull;
    const uint64_t first = w == cw ? cv : bm[w] & (filt[w] ^ flip);
    const uint64_t m = first & (~0ull << (from & 63));
    if (m) {
        cw = w;
        cv = first;
        const P p = (w << 6) + ctz64(m);
        return p < limit ? p : limit;
    }
    for (++w; w < wend && w < (from >> 6) + 3; ++w) {
        const uint64_t x = bm[w] & (filt[w] ^ flip);
        if (x) {
            cw = w;
            cv = x;
            const P p = (w << 6) + ctz64(x);
            return p < limit ? p : limit;
        }
    }
    for (; w < wend; w += 4) {
        const uint64_t a = bm[w] & (filt[w] ^ flip);
        const uint64_t b = w + 1 < wend ? bm[w + 1] & (filt[w + 1] ^ flip) : 0;
        const uint64_t c = w + 2 < wend ? bm[w + 2] & (filt[w + 2] ^ flip) : 0;
        const uint64_t d = w + 3 < wend ? bm[w + 3] & (filt[w + 3] ^ flip) : 0;
        if (a | b | c | d) {
            const P p = first_of4<P>(w, a, b, c, d, limit);
            cw = w + (a ? 0 : (b ? 1 : (c ? 2 : 3)));
            cv = a ? a : (b ? b : (c ? c : d));
            return p;
        }
    }
    return limit;
}

// Last set bit of `bm` at a position in (floor, from], or -1; `first` is
// bm[from >> 6] (read only when from > floor).
template <typename P>
GPJ_HD P prev_bit(const uint64_t* bm, uint64_t first, P from, P floor) {
    if (from <= floor) return -1;
    P w = from >> 6;
    uint64_t m = first & (~0ull >> (63 - (from & 63)));
    for (;;) {
        if (m) {
            const P k = (w << 6) + 63 - clz64(m);
            return k > floor ? k : -1;
        }
        if ((w << 6) <= floor + 1) return -1;
        --w;
        m = bm[w];
    }
}

template <typename P>
GPJ_HD P prev_bit(const uint64_t* bm, P from, P floor) {
    return from <= floor ? -1 : prev_bit<P>(bm, bm[from >> 6], from, floor);
}

GPJ_HD uint32_t read_varint(const uint8_t* ir, int& pc) {
    uint32_t v = 0;
    int shift = 0;
    uint32_t b;
    while ((b = ir[pc++]) & 0x80u) {
        v |= (b & 0x7Fu) << shift;
        shift += 7;
    }
    return v | (b << shift);
}

// Per-level state of the interpreter: level_ends[k] (the end of the value
// entered at level k, -1 unknown) and current_index[k] (the array element
// counter, -1 before the array's '[' is reached).
//
// In registers/local memory, for every level a query may reach, in the
// interpreter's position type P.
template <typename P>
struct LocalLevelsT {
    P ends[kLevelSlots];
    P index[kLevelSlots];
    GPJ_HD void reset(P line_end) {
        ends[0] = line_end;
#pragma unroll
        for (int k = 1; k < kLevelSlots; k++) ends[k] = -1;
#pragma unroll
        for (int k = 0; k < kLevelSlots; k++) index[k] = -1;
    }
    GPJ_HD P end(int k) const { return ends[k]; }
    GPJ_HD void set_end(int k, P v) { ends[k] = v; }
    GPJ_HD P idx(int k) const { return index[k]; }
    GPJ_HD void set_idx(int k, P v) { index[k] = v; }
};
using LocalLevels = LocalLevelsT<int64_t>;

// In registers, for queries that go at most D - 1 levels down (a validated
// query's level is in [0, D) at every step): the arrays are only ever
// indexed by unrolled loops with constant indices, so they stay in
// registers; an access costs D selects instead of a local-memory round trip.
template <int D, typename P>
struct RegLevelsT {
    P ends[D];
    P index[D];
    GPJ_HD void reset(P line_end) {
        ends[0] = line_end;
#pragma unroll
        for (int k = 1; k < D; k++) ends[k] = -1;
#pragma unroll
        for (int k = 0; k < D; k++) index[k] = -1;
    }
    GPJ_HD P end(int k) const {
        P v = -1;
#pragma unroll
        for (int i = 0; i < D; i++) v = i == k ? ends[i] : v;
        return v;
    }
    GPJ_HD void set_end(int k, P v) {
#pragma unroll
        for (int i = 0; i < D; i++) ends[i] = i == k ? v : ends[i];
    }
    GPJ_HD P idx(int k) const {
        P v = -1;
#pragma unroll
        for (int i = 0; i < D; i++) v = i == k ? index[i] : v;
        return v;
    }
    GPJ_HD void set_idx(int k, P v) {
#pragma unroll
        for (int i = 0; i < D; i++) index[i] = i == k ? v : index[i];
    }
};

// Level slots a query needs: one more than its deepest level, rounded up to
// the register-state sizes the kernels are built for.
GPJ_HD int level_slots_for_depth(int depth) { return depth <= 4 ? 5 : (depth <= 8 ? 9 : kLevelSlots); }

// In caller-provided storage (e.g. shared memory, entries `stride` apart),
// as 32-bit offsets from the line start: for lines shorter than 2 GiB and
// queries no deeper than `slots - 1` levels.
struct PackedLevels {
    int32_t* ends;
    int32_t* index;
    int stride;
    int slots;
    int64_t origin;
    static constexpr int32_t kUnset = INT32_MIN;
    GPJ_HD void reset(int64_t line_end) {
        ends[0] = static_cast<int32_t>(line_end - origin);
        for (int k = 1; k < slots; k++) ends[k * stride] = kUnset;
        for (int k = 0; k < slots; k++) index[k * stride] = -1;
    }
    GPJ_HD int64_t end(int k) const {
        const int32_t v = ends[k * stride];
        return v == kUnset ? -1 : origin + v;
    }
    GPJ_HD void set_end(int k, int64_t v) { ends[k * stride] = v < 0 ? kUnset : static_cast<int32_t>(v - origin); }
    GPJ_HD int64_t idx(int k) const { return index[k * stride]; }
    GPJ_HD void set_idx(int k, int64_t v) { index[k * stride] = static_cast<int32_t>(v); }
};

// How the interpreter scans: one thread alone (SeqScan), or the 32 lanes of
// a warp together on one line (WarpScan, query_kernel.cu), every lane
// holding the same interpreter state.
struct SeqScan {
    template <typename P>
    GPJ_HD static P next(const uint64_t* bm, P from, P limit, P& cw, uint64_t& cv) {
        return next_bit<P>(bm, from, limit, cw, cv);
    }
    template <typename P>
    GPJ_HD static P next_filtered(const uint64_t* bm, const uint64_t* filt, bool invert, P from, P limit, P& cw,
                                  uint64_t& cv) {
        return next_bit_filtered<P>(bm, filt, invert, from, limit, cw, cv);
    }
    template <typename P>
    GPJ_HD static P skip(const uint8_t* file, P j, P hi) {
        return skip_ws<P>(file, j, hi);
    }
    GPJ_HD static void store(int64_t* res, int64_t k, int64_t v) { res[k] = v; }
};

// Runs validated bytecode `ir` on the line [line_start, line_end) and writes
// (start, end) pairs to res[2*k], res[2*k+1] for the k-th STORE_RESULT.
// res must hold -1 on entry.  Returns kLineDeferred when the view ends
// before the line's evaluation does (`skip_end`: what a whitespace skip that
// reaches `hi` returns).  Positions are of type P and relative to `base`
// (added to the stored results); `file`, `string_index`, `levels` and
// `colon` are rebased to match.  `lv` holds the per-level state.
template <typename P, typename Levels, typename Scan = SeqScan>
GPJ_HD int run_line_core(const uint8_t* file, P n, P hi, int skip_end, const uint64_t* string_index,
                         const uint64_t* levels, int64_t level_size, const uint64_t* colon, P line_start,
                         P line_end, const uint8_t* ir, int64_t* res, int64_t base, Levels& lv, int& stored) {
    lv.reset(line_end);

    int pc = 0, cur = 0, result_index = 0;
    stored = 0;
    uint8_t type = 0xFF;
    P want_len = 0;
    int64_t want_index = -1;
    const uint8_t* want = nullptr;
    bool execute = true;

    P j = line_start;
    // the search state: j came from next_bit (so it is a structural bit of
    // level cur), and the bitmap word next_bit found it in
    bool found = false;
    P cw = -1;
    uint64_t cv = 0;
    P cend = lv.end(cur);  // lv.end(cur), kept while searching (only opcodes change it)
    P cidx = -1;           // lv.idx(cur) during an index search, written back at its match
    while (j < cend && j < n) {
        const bool ran = execute;
        while (execute) {
            type = ir[pc++];
            switch (type) {
                case 0:  // END
                    return kLineDone;
                case 1: {  // STORE_RESULT (find_value.cu:59-82)
                    j = Scan::template skip<P>(file, j, hi);  // [bounded] stops at end of file
                    if (j >= hi && skip_end) return kLineDeferred;
                    const P e = lv.end(cur);
                    Scan::store(res, 2 * result_index, base + j);
                    Scan::store(res, 2 * result_index + 1, e < 0 ? -1 : base + e);
                    stored = ++result_index;
                    break;
                }
                case 2:  // MOVE_UP (:83-90)
                    if (lv.end(cur) < 0) return kLineDone;  // [bounded] would continue at j=-1
                    j = lv.end(cur);
                    lv.set_end(cur, -1);
                    --cur;
                    break;
                case 3: {  // MOVE_DOWN (:91-111): end of the value = next structural one level up
                    ++cur;
                    if (lv.end(cur) == -1) {
                        const P lim = lv.end(cur - 1);
                        P mw = -1;
                        uint64_t mv = 0;
                        const P m = Scan::template next<P>(levels + level_size * (cur - 1), j + 1, lim, mw, mv);
                        if (m < lim) lv.set_end(cur, m);
                    }
                    break;
                }
                case 4:  // MOVE_TO_KEY (:112-130)
                    want_len = static_cast<P>(read_varint(ir, pc));
                    want = ir + pc;
                    pc += static_cast<int>(want_len);
                    execute = false;
                    break;
                case 5:  // MOVE_TO_INDEX (:131-169)
                    want_index = read_varint(ir, pc);
                    if (lv.idx(cur) == -1) {
                        j = Scan::template skip<P>(file, j, hi);  // [bounded] only whitespace may precede '['
                        if (j >= hi) return skip_end;
                        if (file[j] != '[') return kLineDone;
                        lv.set_idx(cur, 0);
                    }
                    if (want_index == 0) {
                        ++j;
                        execute = true;
                    } else {
                        execute = false;
                        cidx = lv.idx(cur);
                    }
                    break;
                case 6: {  // EXPRESSION_STRING_EQUALS (:170-210)
                    want_len = static_cast<P>(read_varint(ir, pc));
                    want = ir + pc;
                    pc += static_cast<int>(want_len);
                    j = Scan::template skip<P>(file, j, hi);  // [bounded]
                    if (j >= hi && skip_end) return kLineDeferred;
                    if (lv.end(cur) - j != want_len) return kLineDone;
                    for (P k = 0; k < want_len; k++)
                        if (want[k] != file[j + k]) return kLineDone;
                    break;
                }
                default:
                    return kLineDone;
            }
        }
        if (ran) cend = lv.end(cur);

        // Searching: j is a candidate position ([bounded] only inside the file).
        if (j < hi) {
            const uint64_t* bits = levels + level_size * cur;
            const bool structural = found || ((bits[j >> 6] >> (j & 63)) & 1u);
            const uint8_t at = file[j];
            if (type == 4) {  // key match at a structural ':' (:225-251)
                // Loads that do not depend on each other are issued together:
                // the string-index word before j, and the byte where the key's
                // opening quote is when the key ends right before the ':'
                // (the usual layout), checked against the real position below.
                const uint64_t sw = j > line_start ? string_index[(j - 1) >> 6] : 0;
                const int64_t guess = static_cast<int64_t>(j) - 2 - want_len;
                const uint8_t at_guess = guess >= line_start ? file[guess] : 0;
                if (structural && at == ':') {
                    const P string_end = prev_bit<P>(string_index, sw, j - 1, line_start);
                    const int64_t string_start = static_cast<int64_t>(string_end) - want_len;
                    if (string_start >= line_start &&
                        (string_start == guess ? at_guess : file[string_start]) == '"') {
                        bool same = true;
                        for (P k = 0; k < want_len; k++) {
                            if (want[k] != file[string_start + k + 1]) {
                                same = false;
                                break;
                            }
                        }
                        execute = same;
                    }
                }
            } else if (type == 5) {  // index match at a structural ',' (:252-259)
                if (structural && at == ',') {
                    ++cidx;
                    if (want_index == cidx) {
                        lv.set_idx(cur, cidx);
                        execute = true;
                    }
                }
            }
        }
        ++j;
        found = false;
        if (!execute) {
            // Nothing happens until the next structural bit of this level.
            const P lim = cend < n ? cend : n;
            if (j < lim) {
                if (colon)
                    j = Scan::template next_filtered<P>(levels + level_size * cur, colon, type != 4, j, lim, cw, cv);
                else
                    j = Scan::template next<P>(levels + level_size * cur, j, lim, cw, cv);
                found = j < lim;
            }
        } else {
            cw = -1;  // opcodes run next and may change the level
        }
    }
    return kLineDone;
}

// The interpreter on a view's positions as they are (64-bit), with the
// per-level state in `lv` (LocalLevels, PackedLevels); res must hold -1 on
// entry (only the stored results are written).
template <typename Levels>
GPJ_HD int run_line_with(const LineView& v, int64_t line_start, int64_t line_end, const uint8_t* ir,
                         int64_t* res, Levels& lv) {
    int stored = 0;
    return run_line_core<int64_t>(v.file, v.n, v.hi, v.hi < v.n ? kLineDeferred : kLineDone, v.string_index,
                                  v.levels, v.level_size, v.colon, line_start, line_end, ir, res, 0, lv, stored);
}

// Largest line-relative position the 32-bit interpreter handles.
constexpr int64_t kRelLimit = (1ll << 31) - 4096;

// The interpreter in 64-bit positions with the level state in local memory,
// for lines the 32-bit form cannot hold; a separate function, so that its
// state does not add to the registers of the 32-bit form's caller.  Writes
// every one of the res_len entries once.
#ifdef __CUDACC__
static __host__ __device__ __noinline__
#else
static __attribute__((noinline))
#endif
int run_line_wide(const LineView& v, int64_t line_start, int64_t line_end, const uint8_t* ir, int64_t* res,
                  int64_t res_len) {
    LocalLevels lv;
    int stored = 0;
    const int r = run_line_core<int64_t>(v.file, v.n, v.hi, v.hi < v.n ? kLineDeferred : kLineDone, v.string_index,
                                         v.levels, v.level_size, v.colon, line_start, line_end, ir, res, 0, lv,
                                         stored);
    for (int64_t k = 2 * static_cast<int64_t>(stored); k < res_len; k++) res[k] = -1;
    return r;
}

// run_line_with with positions relative to the line's first 64-byte word
// in 32 bits (the usual case: half the integer work per step) and the
// per-level state in registers for queries whose level stays below D.
// Every one of the res_len entries is written once: the stored results,
// then -1 for the slots the line did not reach (res need not be
// initialised).  Lines whose end lies more than rel_limit (<= kRelLimit)
// bytes past that word run in 64 bits; a whitespace skip that reaches
// rel_limit (bytes past it exist) stops there and the line is evaluated
// again in 64 bits.  With a skip_bound, a whitespace skip that runs more
// than skip_bound bytes past the line's end (into the blank lines after it)
// stops there too and run_line returns kLineLong, with res partly written,
// for the caller to evaluate the line again (a warp each, query_kernel.cu).
template <int D = kLevelSlots>
GPJ_HD int run_line(const LineView& v, int64_t line_start, int64_t line_end, const uint8_t* ir, int64_t* res,
                    int64_t res_len, int64_t rel_limit = kRelLimit, int64_t skip_bound = -1) {
    const int64_t base = line_start & ~static_cast<int64_t>(63);
    int stored = 0;
    if (line_end - base <= rel_limit) {
        const int64_t lim =
            skip_bound >= 0 && line_end - base + skip_bound < rel_limit ? line_end - base + skip_bound : rel_limit;
        const bool clamped = v.hi - base > lim;
        const int32_t hi = static_cast<int32_t>(clamped ? lim : v.hi - base);
        const int32_t n = static_cast<int32_t>(v.n - base > rel_limit ? rel_limit : v.n - base);
        const int skip_end = clamped || v.hi < v.n ? kLineDeferred : kLineDone;
        const int64_t w = base >> 6;
        RegLevelsT<D, int32_t> lv;
        const int r = run_line_core<int32_t>(v.file + base, n, hi, skip_end, v.string_index + w, v.levels + w,
                                             v.level_size, v.colon ? v.colon + w : nullptr,
                                             static_cast<int32_t>(line_start - base),
                                             static_cast<int32_t>(line_end - base), ir, res, base, lv, stored);
        if (r != kLineDeferred || !clamped || v.hi < v.n) {
            for (int64_t k = 2 * static_cast<int64_t>(stored); k < res_len; k++) res[k] = -1;
            return r;
        }
        if (skip_bound >= 0) return kLineLong;
    }
    return run_line_wide(v, line_start, line_end, ir, res, res_len);
}

// Deepest level a validated query's bytecode reaches (its MOVE_DOWNs).
GPJ_HD int bytecode_depth(const uint8_t* ir) {
    int pc = 0, level = 0, deepest = 0;
    for (;;) {
        const uint8_t op = ir[pc++];
        if (op == 0 || op > 6) return deepest;
        if (op == 2) --level;
        if (op == 3 && ++level > deepest) deepest = level;
        if (op == 4 || op == 6) {
            const uint32_t len = read_varint(ir, pc);
            pc += static_cast<int>(len);
        }
        if (op == 5) read_varint(ir, pc);
    }
}

// run_line with the register state sized for queries no deeper than `depth`
// (the sizes the kernels are instantiated for).
GPJ_HD int run_line_depth(int depth, const LineView& v, int64_t line_start, int64_t line_end, const uint8_t* ir,
                          int64_t* res, int64_t res_len, int64_t rel_limit = kRelLimit, int64_t skip_bound = -1) {
    switch (level_slots_for_depth(depth)) {
        case 5:
            return run_line<5>(v, line_start, line_end, ir, res, res_len, rel_limit, skip_bound);
        case 9:
            return run_line<9>(v, line_start, line_end, ir, res, res_len, rel_limit, skip_bound);
        default:
            return run_line<kLevelSlots>(v, line_start, line_end, ir, res, res_len, rel_limit, skip_bound);
    }
}

}  // namespace gpj
