// Test-only CPU harness: runs the device code's per-word arithmetic
// (gpjson_b200/csrc/word_ops.cuh) and line interpreter (interp.cuh) on the
// host, in the same tile/word decomposition the index kernel uses, so the
// test suite can compare them with the oracle without a GPU; and the C
// ABI's host I/O (host_io.h).  It is built by tests/conftest.py and never
// used by the library.
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../gpjson_b200/csrc/host_io.h"
#include "../../gpjson_b200/csrc/interp.cuh"
#include "../../gpjson_b200/csrc/query_items.cuh"
#include "../../gpjson_b200/csrc/word_ops.cuh"

using namespace gpj;

namespace {
constexpr int64_t kTileBytes = 16384;
constexpr int kWordsPerTile = kTileBytes / 64;

uint32_t load_u32(const uint8_t* f, int64_t n, int64_t pos) {
    uint32_t v = 0;
    for (int b = 0; b < 4; b++) {
        const int64_t p = pos + b;
        if (p < n) v |= static_cast<uint32_t>(f[p]) << (8 * b);
    }
    return v;
}

int backslash_run_parity_before(const uint8_t* f, int64_t pos, int64_t floor) {
    int64_t k = pos - 1, run = 0;
    while (k >= floor && f[k] == '\\') {
        ++run;
        --k;
    }
    return static_cast<int>(run & 1);
}
}  // namespace

extern "C" {

// Mirrors the index kernel: per tile, word summaries with a local string
// state of 0, an exclusive compose-scan inside the tile, a sequential prefix
// over tiles (the kernel's look-back), then the final masks per word.
int64_t hs_build_index(const uint8_t* f, int64_t n, int num_levels, uint64_t* str_out,
                       uint64_t* lvl_out, int64_t* nl_out, int64_t nl_cap) {
    const int64_t level_size = (n + 63) / 64;
    const int64_t ntiles = (n + kTileBytes - 1) / kTileBytes;
    int s_state = 0;
    int64_t d_state = -1, nl_state = 0;
    if (nl_cap > 0) nl_out[0] = 0;
    std::vector<ClassMasks> masks(kWordsPerTile);
    std::vector<uint64_t> esc(kWordsPerTile), p0(kWordsPerTile);
    std::vector<Span> excl(kWordsPerTile);
    for (int64_t t = 0; t < ntiles; t++) {
        const int64_t tile_start = t * kTileBytes;
        const int tile_parity = backslash_run_parity_before(f, tile_start, 0);
        Span acc = span_identity();
        for (int w = 0; w < kWordsPerTile; w++) {
            const int64_t ws = tile_start + 64 * w;
            uint32_t v[16];
            for (int k = 0; k < 16; k++) v[k] = ws < n ? load_u32(f, n, ws + 4 * k) : 0;
            masks[w] = classify64(v);
            // escape carry: backslash run inside the tile, then before it
            int64_t k = ws - 1, run = 0;
            while (k >= tile_start && f[k] == '\\') {
                ++run;
                --k;
            }
            uint32_t cin = static_cast<uint32_t>(run & 1);
            if (k < tile_start) cin ^= static_cast<uint32_t>(tile_parity);
            uint32_t cout;
            const uint64_t e = escaped_mask(masks[w].backslash, cin, &cout);
            const uint64_t qr = masks[w].quote & ~e;
            p0[w] = prefix_xor(qr);
            Span sp;
            sp.q = popc64(qr) & 1;
            sp.dd0 = popc64(masks[w].open & ~p0[w]) - popc64(masks[w].close & ~p0[w]);
            sp.ddt = popc64(masks[w].open) - popc64(masks[w].close);
            sp.nl = popc64(masks[w].newline);
            excl[w] = acc;
            acc = span_compose(acc, sp);
        }
        // tile prefix (state before the tile) is (s_state, d_state, nl_state)
        for (int w = 0; w < kWordsPerTile; w++) {
            const int64_t ws = tile_start + 64 * w;
            if (ws >= n) break;
            const int64_t word = ws / 64;
            const int s_w = s_state ^ excl[w].q;
            const int64_t d_w = d_state + (s_state ? (excl[w].ddt - excl[w].dd0) : excl[w].dd0);
            uint64_t in_str = p0[w] ^ (s_w ? ~0ull : 0ull);
            const int64_t valid = n - ws < 64 ? n - ws : 64;
            if (valid < 64) in_str &= (1ull << valid) - 1;
            str_out[word] = in_str;
            uint64_t lv[16];
            split_levels<16>(masks[w].open & ~in_str, masks[w].close & ~in_str,
                             masks[w].structural & ~in_str, d_w, lv);
            for (int l = 0; l < num_levels; l++) lvl_out[l * level_size + word] = lv[l];
            int64_t idx = 1 + nl_state + excl[w].nl;
            uint64_t nm = masks[w].newline;
            while (nm) {
                const int p = ctz64(nm);
                if (idx < nl_cap) nl_out[idx] = ws + p;
                ++idx;
                nm &= nm - 1;
            }
        }
        // apply the tile aggregate
        const int s_old = s_state;
        s_state ^= acc.q;
        d_state += s_old ? (acc.ddt - acc.dd0) : acc.dd0;
        nl_state += acc.nl;
    }
    return nl_state + 1;
}

// Mirrors the line-parallel kernel (index_lines.cu): per tile, the lines
// starting in it are indexed from the NDJSON line-start state (outside
// strings, level -1), continuing past the tile end to the first newline;
// words are written by the tile whose range holds their first byte.
// Returns the line count, or -1 when a line does not end in the line-start
// state (the kernel then defers to the exact kernel).
int64_t hs_build_index_lines(const uint8_t* f, int64_t n, int num_levels, uint64_t* str_out,
                             uint64_t* lvl_out, int64_t* nl_out, int64_t nl_cap) {
    const int64_t level_size = (n + 63) / 64;
    const int64_t ntiles = (n + kTileBytes - 1) / kTileBytes;
    int64_t nl_before = 0;
    bool irregular = false;
    if (nl_cap > 0) nl_out[0] = 0;
    for (int64_t t = 0; t < ntiles; t++) {
        const int64_t ts = t * kTileBytes, te = std::min(n, ts + kTileBytes);
        int64_t a = -1;
        for (int64_t i = ts; i < te; i++)
            if (f[i] == '\n') {
                if (a < 0) a = i;
                if (1 + nl_before < nl_cap) nl_out[1 + nl_before] = i;
                ++nl_before;
            }
        if (t == 0) a = 0;
        if (a < 0) continue;
        int64_t b = te;
        while (b < n && f[b] != '\n') ++b;
        // b == te when the tile ends at a newline or at the end of the file
        int s = 0;
        int64_t d = -1;
        uint32_t esc = 0;
        for (int64_t ws = (a / 64) * 64; ws < b || (ws < n && ws < ((b + 63) / 64) * 64); ws += 64) {
            if (ws >= n) break;
            uint32_t v[16];
            for (int k = 0; k < 16; k++) v[k] = load_u32(f, n, ws + 4 * k);
            ClassMasks m = classify64(v);
            uint64_t keep = ~0ull;
            if (a > ws) keep &= ~((1ull << (a - ws)) - 1);
            if (n - ws < 64) keep &= (1ull << (n - ws)) - 1;
            m.backslash &= keep, m.quote &= keep, m.newline &= keep, m.open &= keep, m.close &= keep,
                m.structural &= keep;
            uint32_t cout;
            const uint64_t e = escaped_mask(m.backslash, esc, &cout);
            esc = cout;
            const uint64_t qr = m.quote & ~e;
            const uint64_t in_str = (prefix_xor(qr) ^ (s ? ~0ull : 0ull)) & keep;
            const uint64_t open = m.open & ~in_str, close = m.close & ~in_str;
            // '\n' in (a, b]: must be outside strings at level -1
            uint64_t check = m.newline;
            if (a >= ws && a < ws + 64) check &= ~(1ull << (a - ws));
            if (b < ws + 64 && b >= ws) check &= (b == ws + 63) ? ~0ull : ((2ull << (b - ws)) - 1);
            else if (b < ws) check = 0;
            for (uint64_t c = check; c; c &= c - 1) {
                const int bit = ctz64(c);
                const uint64_t below = (1ull << bit) - 1;
                if ((in_str >> bit) & 1) irregular = true;
                if (d + popc64(open & below) - popc64(close & below) != -1) irregular = true;
            }
            if (ws >= a && ws < b) {
                str_out[ws / 64] = in_str;
                uint64_t lv[16];
                split_levels<16>(open, close, m.structural & ~in_str, d, lv);
                for (int l = 0; l < num_levels; l++) lvl_out[l * level_size + ws / 64] = lv[l];
            }
            d += popc64(open) - popc64(close);
            s = (popc64(qr) & 1) ? !s : s;
        }
    }
    return irregular ? -1 : nl_before + 1;
}

// Runs each query's bytecode on every line with the device interpreter.
// out: [nq][lines][slots][2], filled with -1 here.  `colon` (may be null)
// is the bitmap of ':' outside strings that the fused kernel's key searches
// jump along; `packed` = 1 selects the 32-bit level state the fused kernel
// keeps in shared memory, 2 the line-relative 32-bit interpreter with a
// 64-byte limit (so that its 64-bit fallbacks run), 3 the register state of
// the deepest size (0 sizes it by the query's depth, as the kernels do),
// 4 that with a whitespace-skip bound (the kernels' hand-over of long skips).
// Slots the interpreter does not reach are written -1 by it (run_line) or
// were -1 before (PackedLevels).
void hs_find_values(const uint8_t* f, int64_t n, const int64_t* nl, int64_t lines,
                    const uint64_t* str, const uint64_t* lvl, int nq, const uint8_t* const* irs,
                    int slots, int64_t* out, const uint64_t* colon, int packed) {
    LineView v{f, n, str, lvl, (n + 63) / 64, n, colon};
    const int64_t per_query = lines * slots * 2;
    for (int64_t k = 0; k < per_query * nq; k++) out[k] = -1;
    int32_t ends[kLevelSlots], index[kLevelSlots];
    for (int q = 0; q < nq; q++) {
        for (int64_t i = 0; i < lines; i++) {
            const int64_t start = nl[i];
            const int64_t end = i + 1 < lines ? nl[i + 1] : n;
            int64_t* res = out + q * per_query + i * slots * 2;
            if (packed == 1) {
                PackedLevels lv{ends, index, 1, kLevelSlots, start};
                run_line_with(v, start, end, irs[q], res, lv);
            } else if (packed == 0) {
                for (int k = 0; k < slots * 2; k++) res[k] = 7;  // written again by run_line
                run_line_depth(bytecode_depth(irs[q]), v, start, end, irs[q], res, slots * 2);
            } else if (packed == 4) {
                // a skip bound of 16 bytes past the line: lines that skip further
                // are evaluated again by the 64-bit interpreter, as the kernels
                // hand them to a warp
                for (int k = 0; k < slots * 2; k++) res[k] = 7;
                if (run_line_depth(bytecode_depth(irs[q]), v, start, end, irs[q], res, slots * 2, kRelLimit, 16) ==
                    kLineLong)
                    run_line_wide(v, start, end, irs[q], res, slots * 2);
            } else {
                for (int k = 0; k < slots * 2; k++) res[k] = 7;
                run_line<kLevelSlots>(v, start, end, irs[q], res, slots * 2, packed == 2 ? 64 : kRelLimit);
            }
        }
    }
}

// The byte classes of `words` 64-byte words: out[7 * w + c] = class c
// (backslash, quote, newline, open, close, structural, colon) of word w.
void hs_classify(const uint8_t* bytes, int64_t words, uint64_t* out) {
    for (int64_t w = 0; w < words; w++) {
        uint32_t v[16];
        std::memcpy(v, bytes + 64 * w, 64);
        const ClassMasks m = classify64(v);
        const uint64_t c[7] = {m.backslash, m.quote, m.newline, m.open, m.close, m.structural, m.colon};
        for (int k = 0; k < 7; k++) out[7 * w + k] = c[k];
    }
}

// Escape-mask check on one word against a byte loop.
uint64_t hs_escaped_mask(uint64_t bs, uint32_t cin, uint32_t* cout) {
    return escaped_mask(bs, cin, cout);
}

// The find_value kernels' item numbering: for items [0, query_items) of a
// file, writes (line, query) of each real item to pairs[] (in item order)
// and returns how many there were.
int64_t hs_query_items(int64_t item_begin, int64_t num_lines, int num_queries, int64_t stride, int64_t* pairs) {
    const int64_t items = query_items(num_lines, num_queries);
    int64_t count = 0;
    for (int64_t k = 0; k < items; k++) {
        int64_t line;
        int q;
        if (query_item(k, item_begin, num_lines, num_queries, stride, &line, &q)) {
            pairs[2 * count] = line;
            pairs[2 * count + 1] = q;
            ++count;
        }
    }
    return count;
}

// Reads ranges [pos[i], pos[i] + len[i]) of `path` back to back into dst
// through one gpj::SliceReader of `threads` threads; returns how many
// ranges were read before the first failure (-1: the file does not open).
int hs_read_ranges(const char* path, uint8_t* dst, const int64_t* pos, const int64_t* len, int ranges, int threads) {
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return -1;
    int done = 0;
    {
        gpj::SliceReader reader(fd, threads);
        for (; done < ranges; done++) {
            if (!reader.read(dst, pos[done], static_cast<size_t>(len[done]))) break;
            dst += len[done];
        }
    }
    ::close(fd);
    return done;
}

// gpj::ResultBuffers, one instance per test.
void* hs_rb_new() { return new gpj::ResultBuffers; }
void hs_rb_delete(void* b) { delete static_cast<gpj::ResultBuffers*>(b); }
int64_t* hs_rb_take(void* b, uint64_t count, uint64_t* cap) {
    size_t c = 0;
    int64_t* p = static_cast<gpj::ResultBuffers*>(b)->take(count, &c);
    *cap = c;
    return p;
}
void hs_rb_give(void* b, int64_t* p, uint64_t cap) { static_cast<gpj::ResultBuffers*>(b)->give(p, cap); }
uint64_t hs_rb_keep_elems() { return gpj::ResultBuffers::kKeepElems; }

}  // extern "C"
