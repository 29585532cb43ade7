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

enum LineStatus : int { kLineDone = 0, kLineDeferred = 1 };

GPJ_HD bool is_ws(uint8_t c) { return c == '\n' || c == '\r' || c == '\t' || c == ' '; }

// First set bit of `bm` at a position in [from, limit), or `limit`.  After
// the first three words, four words are loaded per step (independent loads,
// so a long jump waits for a quarter of the dependent memory round trips);
// only words holding positions below `limit` are read.
GPJ_HD int64_t first_of4(int64_t w, uint64_t a, uint64_t b, uint64_t c, uint64_t d, int64_t limit) {
    int64_t base = w;
    uint64_t x = a;
    if (!a) {
        base = b ? w + 1 : (c ? w + 2 : w + 3);
        x = b ? b : (c ? c : d);
    }
    const int64_t p = (base << 6) + ctz64(x);
    return p < limit ? p : limit;
}

// `cw`/`cv`: a word of bm the caller already holds (index, value; cw = -1
// for none), used instead of reloading it; on return they hold the word the
// result was found in.
GPJ_HD int64_t next_bit(const uint64_t* bm, int64_t from, int64_t limit, int64_t& cw, uint64_t& cv) {
    if (from >= limit) return limit;
    int64_t w = from >> 6;
    const int64_t wend = ((limit - 1) >> 6) + 1;
    const uint64_t first = w == cw ? cv : bm[w];
    const uint64_t m = first & (~0ull << (from & 63));
    if (m) {
        cw = w;
        cv = first;
        const int64_t p = (w << 6) + ctz64(m);
        return p < limit ? p : limit;
    }
    // the next two words one at a time (most jumps end there), then four per step
    for (++w; w < wend && w < (from >> 6) + 3; ++w) {
        const uint64_t x = bm[w];
        if (x) {
            cw = w;
            cv = x;
            const int64_t p = (w << 6) + ctz64(x);
            return p < limit ? p : limit;
        }
    }
    for (; w < wend; w += 4) {
        const uint64_t a = bm[w];
        const uint64_t b = w + 1 < wend ? bm[w + 1] : 0;
        const uint64_t c = w + 2 < wend ? bm[w + 2] : 0;
        const uint64_t d = w + 3 < wend ? bm[w + 3] : 0;
        if (a | b | c | d) {
            const int64_t p = first_of4(w, a, b, c, d, limit);
            cw = w + (a ? 0 : (b ? 1 : (c ? 2 : 3)));
            cv = a ? a : (b ? b : (c ? c : d));
            return p;
        }
    }
    return limit;
}

GPJ_HD int64_t next_bit(const uint64_t* bm, int64_t from, int64_t limit) {
    int64_t cw = -1;
    uint64_t cv = 0;
    return next_bit(bm, from, limit, cw, cv);
}

// First position in [from, limit) set in bm and (in `filt`, or not in it
// when `invert`), or `limit`.
GPJ_HD int64_t next_bit_filtered(const uint64_t* bm, const uint64_t* filt, bool invert, int64_t from,
                                 int64_t limit) {
    if (from >= limit) return limit;
    int64_t w = from >> 6;
    const int64_t wend = ((limit - 1) >> 6) + 1;
    const uint64_t flip = invert ? ~0ull : 0ull;
    const uint64_t m = bm[w] & (filt[w] ^ flip) & (~0ull << (from & 63));
    if (m) {
        const int64_t p = (w << 6) + ctz64(m);
        return p < limit ? p : limit;
    }
    for (++w; w < wend && w < (from >> 6) + 3; ++w) {
        const uint64_t x = bm[w] & (filt[w] ^ flip);
        if (x) {
            const int64_t p = (w << 6) + ctz64(x);
            return p < limit ? p : limit;
        }
    }
    for (; w < wend; w += 4) {
        const uint64_t a = bm[w] & (filt[w] ^ flip);
        const uint64_t b = w + 1 < wend ? bm[w + 1] & (filt[w + 1] ^ flip) : 0;
        const uint64_t c = w + 2 < wend ? bm[w + 2] & (filt[w + 2] ^ flip) : 0;
        const uint64_t d = w + 3 < wend ? bm[w + 3] & (filt[w + 3] ^ flip) : 0;
        if (a | b | c | d) return first_of4(w, a, b, c, d, limit);
    }
    return limit;
}

// Last set bit of `bm` at a position in (floor, from], or -1; `first` is
// bm[from >> 6] (read only when from > floor).
GPJ_HD int64_t prev_bit(const uint64_t* bm, uint64_t first, int64_t from, int64_t floor) {
    if (from <= floor) return -1;
    int64_t w = from >> 6;
    uint64_t m = first & (~0ull >> (63 - (from & 63)));
    for (;;) {
        if (m) {
            const int64_t k = (w << 6) + 63 - clz64(m);
            return k > floor ? k : -1;
        }
        if ((w << 6) <= floor + 1) return -1;
        --w;
        m = bm[w];
    }
}

GPJ_HD int64_t prev_bit(const uint64_t* bm, int64_t from, int64_t floor) {
    return from <= floor ? -1 : prev_bit(bm, bm[from >> 6], from, floor);
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
// In registers/local memory, for every level a query may reach.
struct LocalLevels {
    int64_t ends[kLevelSlots];
    int64_t index[kLevelSlots];
    GPJ_HD void reset(int64_t line_end) {
        ends[0] = line_end;
#pragma unroll
        for (int k = 1; k < kLevelSlots; k++) ends[k] = -1;
#pragma unroll
        for (int k = 0; k < kLevelSlots; k++) index[k] = -1;
    }
    GPJ_HD int64_t end(int k) const { return ends[k]; }
    GPJ_HD void set_end(int k, int64_t v) { ends[k] = v; }
    GPJ_HD int64_t idx(int k) const { return index[k]; }
    GPJ_HD void set_idx(int k, int64_t v) { index[k] = v; }
};

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

// Runs validated bytecode `ir` on the line [line_start, line_end) and writes
// (start, end) pairs to res[2*k], res[2*k+1] for the k-th STORE_RESULT.
// res must hold -1 on entry.  Returns kLineDeferred when the view ends
// before the line's evaluation does.  `lv` holds the per-level state.
template <typename Levels>
GPJ_HD int run_line_with(const LineView& v, int64_t line_start, int64_t line_end, const uint8_t* ir,
                         int64_t* res, Levels& lv) {
    lv.reset(line_end);

    const uint8_t* file = v.file;
    const int64_t n = v.n;
    const int64_t hi = v.hi;
    const int skip_end = hi < n ? kLineDeferred : kLineDone;
    int pc = 0, cur = 0, result_index = 0;
    uint8_t type = 0xFF;
    int64_t want_len = 0, want_index = -1;
    const uint8_t* want = nullptr;
    bool execute = true;

    int64_t j = line_start;
    // the search state: j came from next_bit (so it is a structural bit of
    // level cur), and the bitmap word next_bit found it in
    bool found = false;
    int64_t cw = -1;
    uint64_t cv = 0;
    int64_t cend = lv.end(cur);  // lv.end(cur), kept while searching (only opcodes change it)
    while (j < cend && j < n) {
        const bool ran = execute;
        while (execute) {
            type = ir[pc++];
            switch (type) {
                case 0:  // END
                    return kLineDone;
                case 1:  // STORE_RESULT (find_value.cu:59-82)
                    while (j < hi && is_ws(file[j])) ++j;  // [bounded] stops at end of file
                    if (j >= hi && skip_end) return kLineDeferred;
                    res[2 * result_index] = j;
                    res[2 * result_index + 1] = lv.end(cur);
                    ++result_index;
                    break;
                case 2:  // MOVE_UP (:83-90)
                    if (lv.end(cur) < 0) return kLineDone;  // [bounded] would continue at j=-1
                    j = lv.end(cur);
                    lv.set_end(cur, -1);
                    --cur;
                    break;
                case 3: {  // MOVE_DOWN (:91-111): end of the value = next structural one level up
                    ++cur;
                    if (lv.end(cur) == -1) {
                        const int64_t lim = lv.end(cur - 1);
                        const int64_t m = next_bit(v.levels + v.level_size * (cur - 1), j + 1, lim);
                        if (m < lim) lv.set_end(cur, m);
                    }
                    break;
                }
                case 4:  // MOVE_TO_KEY (:112-130)
                    want_len = read_varint(ir, pc);
                    want = ir + pc;
                    pc += static_cast<int>(want_len);
                    execute = false;
                    break;
                case 5:  // MOVE_TO_INDEX (:131-169)
                    want_index = read_varint(ir, pc);
                    if (lv.idx(cur) == -1) {
                        for (;;) {  // [bounded] only whitespace may precede '['
                            if (j >= hi) return skip_end;
                            const uint8_t c = file[j];
                            if (c == '[') break;
                            if (!is_ws(c)) return kLineDone;
                            ++j;
                        }
                        lv.set_idx(cur, 0);
                    }
                    if (want_index == 0) {
                        ++j;
                        execute = true;
                    } else {
                        execute = false;
                    }
                    break;
                case 6: {  // EXPRESSION_STRING_EQUALS (:170-210)
                    want_len = read_varint(ir, pc);
                    want = ir + pc;
                    pc += static_cast<int>(want_len);
                    while (j < hi && is_ws(file[j])) ++j;  // [bounded]
                    if (j >= hi && skip_end) return kLineDeferred;
                    if (lv.end(cur) - j != want_len) return kLineDone;
                    for (int64_t k = 0; k < want_len; k++)
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
            const uint64_t* bits = v.levels + v.level_size * cur;
            const bool structural = found || ((bits[j >> 6] >> (j & 63)) & 1u);
            const uint8_t at = file[j];
            if (type == 4) {  // key match at a structural ':' (:225-251)
                // Loads that do not depend on each other are issued together:
                // the string-index word before j, and the byte where the key's
                // opening quote is when the key ends right before the ':'
                // (the usual layout), checked against the real position below.
                const uint64_t sw = j > line_start ? v.string_index[(j - 1) >> 6] : 0;
                const int64_t guess = j - 2 - want_len;
                const uint8_t at_guess = guess >= line_start ? file[guess] : 0;
                if (structural && at == ':') {
                    const int64_t string_end = prev_bit(v.string_index, sw, j - 1, line_start);
                    const int64_t string_start = string_end - want_len;
                    if (string_start >= line_start &&
                        (string_start == guess ? at_guess : file[string_start]) == '"') {
                        bool same = true;
                        for (int64_t k = 0; k < want_len; k++) {
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
                    const int64_t count = lv.idx(cur) + 1;
                    lv.set_idx(cur, count);
                    if (want_index == count) execute = true;
                }
            }
        }
        ++j;
        found = false;
        if (!execute) {
            // Nothing happens until the next structural bit of this level.
            const int64_t lim = cend < n ? cend : n;
            if (j < lim) {
                if (v.colon)
                    j = next_bit_filtered(v.levels + v.level_size * cur, v.colon, type != 4, j, lim);
                else
                    j = next_bit(v.levels + v.level_size * cur, j, lim, cw, cv);
                found = j < lim;
            }
        } else {
            cw = -1;  // opcodes run next and may change the level
        }
    }
    return kLineDone;
}

GPJ_HD int run_line(const LineView& v, int64_t line_start, int64_t line_end, const uint8_t* ir, int64_t* res) {
    LocalLevels lv;
    return run_line_with(v, line_start, line_end, ir, res, lv);
}

}  // namespace gpj
