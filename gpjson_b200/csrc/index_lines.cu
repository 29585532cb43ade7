// Line-parallel structural index for NDJSON on sm_100a, with the JSONPath
// queries evaluated in the same pass (the fast path).
//
// In newline-delimited JSON every line is a complete value, so at each
// '\n' the reference's scan state (Sequential.java:36-128: inside-string
// flag, level counter, escape flag) is (outside, -1, clear) again.  This
// kernel uses that: the CTA that owns a 14 KiB tile builds the index of
// every line that starts in it, starting each line from that state, and runs
// on past the tile end to finish its last line (in the 2 KiB look-ahead
// loaded with the tile, or from device memory for longer lines).  No string or level carry
// crosses tiles, so CTAs depend on each other only through the newline
// count, which a decoupled look-back resolves off the critical path.
//
// The assumption is checked, not trusted: before every '\n' the computed
// state must be (outside, -1).  If any line breaks it (a raw newline inside
// a string, unbalanced brackets, garbage) the kernel flags the input and the
// host rebuilds the index with the exact carry-propagating kernel
// (index_exact.cu), so the output always equals the sequential definition.
//
// Ownership: the CTA of tile t owns the byte range R_t = [a_t, b_t) from the
// first '\n' of the tile (byte 0 for tile 0) to the first '\n' at or after
// the tile end, and writes every bitmap word whose first byte lies in R_t,
// computing all 64 bits of it with its own running state.
//
// Each CTA is a three-stage pipeline over its tiles (tile blockIdx.x, then
// every gridDim.x-th):
//  * copies: 1-D TMA bulk loads of tile + look-ahead (16 KiB) into a ring
//    of byte slots (three here; two in the standalone kernel, whose tiles'
//    bytes nobody reads after the tile's last barrier), issued one tile ahead;
//  * index warps (0-7, one 64-byte word of the slot per thread): classify,
//    resolve escapes and strings, one block scan with a reset at newlines
//    (line starts, newline counts and each word's state at once), split
//    levels, write the index, and leave the final masks of the tile and its
//    look-ahead in one of two mask slots;
//  * line warps (8-11): the newline-count look-back, the newline index, and
//    the find_value interpreter (interp.cuh) on the tile's lines over the
//    shared-memory masks, one (line, query) pair per thread, a warp's lanes
//    on one query.
// The stages hand slots over through mbarriers, so the look-back and the
// queries of tile k overlap the indexing of tile k+1.  Lines the line warps
// cannot evaluate from shared memory are flagged and the host evaluates all
// lines with the find_value kernel instead.
#include <atomic>
#include <cstdint>

#include "device_common.cuh"
#include "index_kernel.h"
#include "interp.cuh"
#include "tile_common.cuh"
#include "word_ops.cuh"

namespace gpj {

namespace {

constexpr int64_t kTile = kLineTileBytes;            // 14 KiB owned per tile
constexpr int kTileWords = kTile / 64;               // 224
constexpr int64_t kExtBytes = 2048;                  // look-ahead loaded with the tile
constexpr int64_t kSlotBytes = kTile + kExtBytes;    // 16 KiB: one word per index thread
constexpr int kSlotWords = kTileWords + kExtBytes / 64;  // 256
static_assert(kSlotWords == 256 && kSlotBytes == kRoundBytes, "one slot word per index thread");
constexpr int kRing = 3;                             // byte slots
constexpr int kMaskSlots = 2;
constexpr int kIndexThreads = 256;                   // warps 0-7
constexpr int kLineThreads = 128;                    // warps 8-11
constexpr int kThreads = kIndexThreads + kLineThreads;
constexpr int kBarIndex = 1;                         // named barrier ids
constexpr int kBarLines = 2;
constexpr int64_t kNone = INT64_MAX;
// Longest run past the tile end a CTA follows to finish its last line; a
// longer line sends the whole input to the exact kernel.  One CTA walks the
// run alone, one round after the other, while the exact kernel spreads a
// line over all its tiles: on inputs with lines of a megabyte (4 GiB,
// lines log-uniform 100 B-1 MiB) the bound of 64 KiB halves the index build
// (31.7 -> 15.1 ms) against one of 8 MiB.
constexpr int64_t kMaxExtension = 64ll << 10;
// Lines of one tile whose starts are kept for the fused queries.
constexpr int kMaxTileLines = 512;
// Bytecode of the fused queries kept in shared memory (else read from
// device memory).
constexpr int kIrBytes = 2048;
constexpr int kIrQueries = 256;
constexpr unsigned long long kPayload48 = (1ull << 48) - 1;

__device__ __forceinline__ void group_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

__device__ __forceinline__ unsigned long long tag48(uint32_t epoch, unsigned long long v) {
    return (static_cast<unsigned long long>(epoch) << 48) | (v & kPayload48);
}
__device__ __forceinline__ bool has_tag(unsigned long long w, uint32_t epoch) {
    return static_cast<uint32_t>(w >> 48) == epoch;
}
__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.volatile.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Number of newlines before tile t (decoupled look-back over per-tile counts,
// eight tiles per lane per step).  Executed by one full warp; lane 0
// publishes the tile's inclusive count.
constexpr int kPerLane = 8;

__device__ int64_t lookback_newlines(unsigned long long* agg, unsigned long long* inc, int64_t t, int64_t count,
                                     uint32_t epoch, unsigned long long* status) {
    const int lane = threadIdx.x & 31;
    int64_t acc = 0;
    int64_t base = t - 1;
    unsigned polls = 0;
    while (base >= 0) {
        unsigned long long a[kPerLane], g[kPerLane];
#pragma unroll
        for (int k = 0; k < kPerLane; k++) {
            const int64_t p = base - kPerLane * lane - k;
            a[k] = p >= 0 ? ld_volatile(inc + p) : 0;
            g[k] = p >= 0 ? ld_volatile(agg + p) : 0;
        }
        int st = 1;  // 0 not ready, 1 all aggregates, 2 inclusive found
        int64_t lane_sum = 0, inc_val = 0;
#pragma unroll
        for (int k = 0; k < kPerLane; k++) {
            if (st != 1) continue;
            const int64_t p = base - kPerLane * lane - k;
            if (p < 0) {
                st = 2;
                inc_val = 0;
            } else if (has_tag(a[k], epoch)) {
                st = 2;
                inc_val = static_cast<int64_t>(a[k] & kPayload48);
            } else if (has_tag(g[k], epoch)) {
                lane_sum += static_cast<int64_t>(g[k] & kPayload48);
            } else {
                st = 0;
            }
        }
        const unsigned inc_mask = __ballot_sync(~0u, st == 2);
        const unsigned bad_mask = __ballot_sync(~0u, st == 0);
        const int first = inc_mask ? __ffs(inc_mask) - 1 : 32;
        const unsigned need = first == 32 ? ~0u : ((2u << first) - 1);  // lanes 0..first
        if (bad_mask & need) {
            ++polls;
            const bool expired =
                polls > kMaxPolls || ((polls & 1023u) == 0 && (ld_acquire(status + 1) & kFatalErrors) != 0);
            if (expired) {
                if (lane == 0) atomicOr(status + 1, kErrLookbackTimeout);
                break;
            }
            __nanosleep(64);
            continue;
        }
        int64_t part = lane <= first ? lane_sum : 0;
        if (lane == first) part += inc_val;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(~0u, part, off);
        acc += part;
        if (first < 32) break;
        base -= 32 * kPerLane;
    }
    if (lane == 0) st_release(inc + t, tag48(epoch, static_cast<unsigned long long>(acc + count)));
    return acc;
}

// What the index warps hand to the line warps about one tile.
struct SlotInfo {
    int64_t a;   // first line start (kNone: no line starts in the tile)
    int64_t b;   // end of the last line
    int64_t hi;  // bytes [tile_start, hi) have final masks in the slot
    int tile_nl;  // newlines in the tile
    int byte_slot;
};

// The tile scan.  A word holding a '\n' starts a line there; in NDJSON
// every line starts outside strings at level -1, so the state after such a
// word is known absolutely from its bytes past its first '\n' (a reset).
// Any other word changes the state relatively: it flips the string state
// with its quote parity and changes the level by d_out when entered outside
// a string, by d_in when entered inside (starting inside a string flips
// every in-string bit of the word; the Span arithmetic of word_ops.cuh).  A
// word's state is that of the last reset before it in the tile carried over
// the words between; composing from the last reset is exact because the
// kernel checks the state at every later '\n' (a mismatch sends the input to
// the exact kernel).
//
// Within a warp the string states come from two ballots (resets, parities)
// and a popcount, and the levels from one shuffle prefix sum carrying both
// variants (entered outside / inside) as biased 16-bit halves; the eight
// warp summaries are combined the same way in the first nine lanes of every
// warp (lane 8 = the state after the whole slot).
struct WarpSum {
    int32_t reset;  // a line of the tile starts in the warp
    int32_t s;      // reset: string state after the warp; else: its quote parity
    int32_t d_out;  // reset: level after the warp; else: level change when entered outside a string
    int32_t d_in;   // no reset: level change when entered inside a string
    int32_t nl;     // newlines: of tile words in the low 16 bits, of look-ahead words above
};

// A word's state at its first byte, and the slot's totals.
struct TileScan {
    int reset;       // a line of the tile starts before the word (s, d valid)
    int s;           // in a string
    int d;           // level
    int nl_before;   // newlines before the word (tile words low 16 bits, look-ahead above)
    int lines_here;  // a line starts in the tile
    int s_end;       // state after the slot's last word
    int d_end;
    int nl_total;    // newlines of the slot, as nl_before
};

template <int LV>
struct FShared {
    // the line warps read a tile's bytes while the next tile is indexed and
    // the one after is copied: three byte slots
    static constexpr int kByteSlots = kRing;
    uint8_t bytes[kByteSlots][kSlotBytes];
    TileFile desc[kRing];  // the file of the tile (by tile number modulo kRing)
    uint64_t str[kMaskSlots][kSlotWords];
    uint64_t colon[kMaskSlots][kSlotWords];
    uint64_t lv[kMaskSlots][LV][kSlotWords];
    uint64_t nlmask[kMaskSlots][kTileWords];
    int32_t nlexcl[kMaskSlots][kTileWords];
    int32_t nlpos[kMaskSlots][kMaxTileLines];
    // interpreter state of the line threads (PackedLevels), level-major
    int32_t lvl_end[LV + 1][kLineThreads];
    int32_t lvl_idx[LV + 1][kLineThreads];
    uint8_t ir[kIrBytes];
    int32_t ir_off[kIrQueries];
    SlotInfo info[kMaskSlots];
    uint64_t lvacc[kTileWarps][LV][32];  // level split of each index warp (split_levels_warp)
    uint64_t full[kRing];   // TMA landed
    uint64_t bfree[kRing];  // line warps done with the bytes
    uint64_t mready[kMaskSlots];
    uint64_t mfree[kMaskSlots];
    Span span_scratch[kTileWarps];
    WarpSum rscan[2][kTileWarps];  // tile scan, alternating between tiles
    int carry_esc;
    int64_t first_line;  // start of the tile's first line (its first '\n')
    int64_t ext_b;       // end of the tile's last line when it ends in the look-ahead
    int64_t long_b;
    int64_t nl_before;
};

// Exclusive compose-scan over the NW * 32 index threads (named barrier).
template <int NW = kTileWarps>
__device__ __forceinline__ Span index_scan_span(Span mine, Span* scratch, Span* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Span incl = mine;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const Span o = shfl_span_up(incl, off);
        if (lane >= off) incl = span_compose(o, incl);
    }
    if (lane == 31) scratch[warp] = incl;
    Span excl = shfl_span_up(incl, 1);
    if (lane == 0) excl = span_identity();
    group_sync(kBarIndex, NW * 32);
    Span prefix = span_identity(), all = span_identity();
#pragma unroll
    for (int w = 0; w < NW; w++) {
        if (w == warp) prefix = all;
        all = span_compose(all, scratch[w]);
    }
    *total = all;
    group_sync(kBarIndex, NW * 32);  // scratch may be reused after this
    return span_compose(prefix, excl);
}

// The tile scan over the NW * 32 index threads in word order (see WarpSum;
// a thread's entry may also stand for several consecutive words); one named
// barrier.  Per word: reset_w (a tile line starts in it), q (its
// string state after the reset, else its quote parity), d_abs (reset: level
// after it), d_out / d_in (no reset: level change entered outside / inside a
// string), nl (as WarpSum::nl).  `sums` (kTileWarps entries) must not be
// reused by the next tile (the caller alternates two).  `start_reset`: a
// line starts at the slot's first byte (the file's first tile).
// kBias: the largest level change of one entry (64 per word it stands for),
// so that every biased entry is >= 0 and 32 of them fit in 16 bits.
template <int NW = kTileWarps, int kBias = 64>
__device__ __forceinline__ TileScan tile_scan(bool reset_w, int q, int d_abs, int d_out, int d_in, int nl,
                                              bool start_reset, WarpSum* sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1;
    // ---- within the warp
    const unsigned b_reset = __ballot_sync(~0u, reset_w);
    const unsigned b_q = __ballot_sync(~0u, q != 0);
    const unsigned before = b_reset & lt;
    const int r = before ? 31 - __clz(before) : 0;  // the last reset lane before this one
    const int s_loc = __popc(b_q & (before ? lt & ~((1u << r) - 1) : lt)) & 1;
    // this word's level change for the words after it, the warp entered outside (a) / inside (b) a string
    int da = 0, db = 0;
    if (!reset_w) {
        da = s_loc ? d_in : d_out;
        db = before ? da : (s_loc ? d_out : d_in);
    }
    const uint32_t mine = static_cast<uint32_t>(da + kBias) | (static_cast<uint32_t>(db + kBias) << 16);
    uint32_t incl = mine;
    int nl_incl = nl;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(~0u, incl, off);
        const int on = __shfl_up_sync(~0u, nl_incl, off);
        if (lane >= off) {
            incl += o;
            nl_incl += on;
        }
    }
    const uint32_t excl = incl - mine;
    const int ea = static_cast<int>(excl & 0xFFFF) - kBias * lane;
    const int eb = static_cast<int>(excl >> 16) - kBias * lane;
    const int a_r = __shfl_sync(~0u, d_abs, r);
    const int pa_r = static_cast<int>(__shfl_sync(~0u, incl, r) & 0xFFFF) - kBias * (r + 1);
    // the warp's summary
    const uint32_t all = __shfl_sync(~0u, incl, 31);
    const int last = b_reset ? 31 - __clz(b_reset) : 0;
    const int a_last = __shfl_sync(~0u, d_abs, last);
    const int pa_last = static_cast<int>(__shfl_sync(~0u, incl, last) & 0xFFFF) - kBias * (last + 1);
    const int nl_warp = __shfl_sync(~0u, nl_incl, 31);
    if (lane == 0) {
        WarpSum w;
        w.reset = b_reset != 0;
        w.nl = nl_warp;
        if (b_reset) {
            w.s = __popc(b_q & ~((1u << last) - 1)) & 1;
            w.d_out = a_last + (static_cast<int>(all & 0xFFFF) - kBias * 32) - pa_last;
            w.d_in = w.d_out;
        } else {
            w.s = __popc(b_q) & 1;
            w.d_out = static_cast<int>(all & 0xFFFF) - kBias * 32;
            w.d_in = static_cast<int>(all >> 16) - kBias * 32;
        }
        sums[warp] = w;
    }
    group_sync(kBarIndex, NW * 32);
    // ---- across the warps: lane w < NW holds warp w's summary, lane NW an empty one
    WarpSum w{0, 0, 0, 0, 0};
    if (lane < NW) w = sums[lane];
    const unsigned c_reset = __ballot_sync(~0u, w.reset != 0);
    const unsigned c_q = __ballot_sync(~0u, w.s != 0);
    const unsigned cb = c_reset & lt;
    const int cr = cb ? 31 - __clz(cb) : 0;
    // state at the start of warp `lane`: from its last reset warp, else from the slot start
    const int cs = __popc(c_q & (cb ? lt & ~((1u << cr) - 1) : lt)) & 1;
    const int cdelta = w.reset ? 0 : (cs ? w.d_in : w.d_out);
    int cincl = cdelta, cnl = w.nl;
#pragma unroll
    for (int off = 1; off <= NW; off <<= 1) {
        const int o = __shfl_up_sync(~0u, cincl, off);
        const int on = __shfl_up_sync(~0u, cnl, off);
        if (lane >= off) {
            cincl += o;
            cnl += on;
        }
    }
    const int c_abs = __shfl_sync(~0u, w.d_out, cr);
    const int c_incl_r = __shfl_sync(~0u, cincl, cr);
    const int c_has = (cb != 0 || start_reset) ? 1 : 0;
    const int cd = cb ? c_abs + (cincl - cdelta) - c_incl_r : (start_reset ? -1 : 0) + (cincl - cdelta);
    const int cnl_excl = cnl - w.nl;
    const int in_has = __shfl_sync(~0u, c_has, warp);
    const int in_s = __shfl_sync(~0u, cs, warp);
    const int in_d = __shfl_sync(~0u, cd, warp);
    const int in_nl = __shfl_sync(~0u, cnl_excl, warp);
    TileScan out;
    if (before) {
        out.reset = 1;
        out.s = s_loc;
        out.d = a_r + ea - pa_r;
    } else {
        out.reset = in_has;
        out.s = in_s ^ s_loc;
        out.d = in_d + (in_s ? eb : ea);
    }
    out.nl_before = in_nl + (nl_incl - nl);
    out.lines_here = __shfl_sync(~0u, c_has, NW);
    out.s_end = __shfl_sync(~0u, cs, NW);
    out.d_end = __shfl_sync(~0u, cd, NW);
    out.nl_total = __shfl_sync(~0u, cnl_excl, NW);
    return out;
}

// Issues the TMA load of [start, start + bytes) into `dst` on `bar` (one thread).
__device__ __forceinline__ void load_slot(const uint8_t* file, int64_t start, int64_t bytes, uint8_t* dst,
                                          uint64_t* bar) {
    const uint32_t bulk = static_cast<uint32_t>(bytes & ~static_cast<int64_t>(15));
    // the last bytes of a file that do not fill 16 go by plain copies, before
    // the arrive, so the threads waiting on `bar` see them too
    for (int64_t i = bulk; i < bytes; i++) dst[i] = file[start + i];
    fence_proxy_async_smem();
    if (bulk > 0) {
        mbar_arrive_expect_tx(bar, bulk);
        tma_load_1d(dst, file + start, bulk, bar);
    } else {
        mbar_arrive(bar);
    }
}

// Loads and classifies the 64-byte word at global position `pos` straight
// from device memory (long extensions that do not fit the slot).
__device__ __forceinline__ ClassMasks classify_global(const uint8_t* file, int64_t n, int64_t pos) {
    uint32_t v[16];
    if (pos + 64 <= n) {
        const uint4* src = reinterpret_cast<const uint4*>(file + pos);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint4 q = __ldg(src + i);
            v[4 * i] = q.x, v[4 * i + 1] = q.y, v[4 * i + 2] = q.z, v[4 * i + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 16; i++) {
            uint32_t x = 0;
            for (int b = 0; b < 4; b++) {
                const int64_t q = pos + 4 * i + b;
                if (q < n) x |= static_cast<uint32_t>(__ldg(file + q)) << (8 * b);
            }
            v[i] = x;
        }
    }
    return classify64(v);
}

// Bits 0..x of a word (x in 0..63).
__device__ __forceinline__ uint64_t bits_upto(int x) { return x >= 63 ? ~0ull : ((2ull << x) - 1); }

// Position of the i-th (from 0) set bit of k, which has more than i set bits.
__device__ __forceinline__ int select_bit(uint64_t k, int i) {
    uint32_t w = static_cast<uint32_t>(k);
    int pos = 0;
    const int c32 = __popc(w);
    if (i >= c32) {
        w = static_cast<uint32_t>(k >> 32);
        pos = 32;
        i -= c32;
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const int c = __popc(w & ((1u << s) - 1));
        if (i >= c) {
            w >>= s;
            pos += s;
            i -= c;
        }
    }
    return pos;
}

// split_levels (word_ops.cuh) for the 32 words of a warp at once.  A word
// is cut into segments of constant level at its bracket cuts (`open |
// close << 1`).  Each word keeps its first segment itself; the segments
// that start at a cut are dealt out over the lanes, one per lane per pass
// (ceil(cuts of the warp / 32) passes), and OR-ed into the owning word's
// level slots in `acc` (this warp's [LV][32] words of shared memory).
// Bracket counts differ a lot between words (most have none, some ten or
// more), so a per-word loop would run as long as the warp's densest word;
// here the warp makes about one pass.  Called by all 32 lanes.
template <int LV>
__device__ __forceinline__ void split_levels_warp(uint64_t open, uint64_t close, uint64_t structural, int64_t depth,
                                                  uint64_t (*acc)[32], uint64_t (&lv)[LV]) {
    const int lane = threadIdx.x & 31;
    const uint64_t close_after = close << 1;
    const uint64_t cuts = open | close_after;
    // a word moves the level by at most 64: clamping keeps "out of range"
    const int d = depth > 128 ? 128 : (depth < -128 ? -128 : static_cast<int>(depth));
    const uint64_t first = cuts & (~cuts + 1);
    const uint64_t seg0 = structural & (first - 1);  // all of it when there is no cut
#pragma unroll
    for (int k = 0; k < LV; k++) acc[k][lane] = d == k ? seg0 : 0ull;
    const int m = popc64(cuts);
    int incl = m;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int o = __shfl_up_sync(~0u, incl, off);
        if (lane >= off) incl += o;
    }
    const int base = incl - m;
    const int total = __shfl_sync(~0u, incl, 31);
    __syncwarp();
    for (int r = 0; r < total; r += 32) {
        const int g = r + lane;  // this lane's cut, numbered across the warp
        int o = 0;               // its word: the last lane whose first cut number is <= g
#pragma unroll
        for (int s = 16; s > 0; s >>= 1)
            if (__shfl_sync(~0u, base, o + s) <= g) o += s;
        const int i = g - __shfl_sync(~0u, base, o);
        const uint64_t k = __shfl_sync(~0u, cuts, o);
        const uint64_t op = __shfl_sync(~0u, open, o);
        const uint64_t ca = __shfl_sync(~0u, close_after, o);
        const uint64_t st = __shfl_sync(~0u, structural, o);
        const int dd = __shfl_sync(~0u, d, o);
        if (g < total) {
            const int x = select_bit(k, i);
            const uint64_t upto = bits_upto(x);
            const uint64_t later = k & ~upto;
            // bytes from the cut up to the next one (or the word end)
            const uint64_t seg = st & ~(upto >> 1) & ((later & (~later + 1)) - 1);
            const int level = dd + popc64(op & upto) - popc64(ca & upto);
            if (seg && level >= 0 && level < LV) atomicOr(reinterpret_cast<unsigned long long*>(&acc[level][o]), static_cast<unsigned long long>(seg));
        }
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < LV; k++) lv[k] = acc[k][lane];
}

// Final masks of one word: checks the '\n' bits in `check`, keeps the word
// in mask slot `ms` at `slot` (>= 0) and writes it to the global index when
// `owned`; a word that is not `active` does nothing.  Called at one place
// by every lane of a warp, so the level split's loop over bracket cuts runs
// once per warp (its trip count is the largest of the lanes').
template <int LV, bool kMasks, class Sh>
__device__ __forceinline__ void finish_word(const IndexParams& p, const TileFile& F, Sh& sh, int ms,
                                            const ClassMasks& m,
                                            uint64_t p0, int s_w, int64_t d_w, int64_t word, bool owned, int slot,
                                            uint64_t valid, uint64_t check, bool active) {
    const uint64_t in_str = (p0 ^ (s_w ? ~0ull : 0ull)) & valid;
    const uint64_t open = m.open & ~in_str, close = m.close & ~in_str;
    if (active && check) {
        // every checked '\n' must be outside strings at level -1
        if (check & in_str) atomicOr(F.status + 1, kErrIrregular);
        uint64_t c = check;
        while (c) {
            const int bit = ctz64(c);
            const uint64_t below = (1ull << bit) - 1;
            const int64_t d = d_w + popc64(open & below) - popc64(close & below);
            if (d != -1) atomicOr(F.status + 1, kErrIrregular);
            c &= c - 1;
        }
    }
    const bool split = active && (owned || slot >= 0);
    const uint64_t keep = split ? ~0ull : 0ull;
    uint64_t lv[LV];
    split_levels_warp<LV>(open & keep, close & keep, m.structural & ~in_str & keep, d_w, sh.lvacc[threadIdx.x >> 5],
                          lv);
    if (!split) return;
    if constexpr (kMasks) {
        if (slot >= 0) {
            sh.str[ms][slot] = in_str;
            sh.colon[ms][slot] = m.colon & ~in_str;
#pragma unroll
            for (int l = 0; l < LV; l++) sh.lv[ms][l][slot] = lv[l];
        }
    }
    if (owned && p.materialize) {
        F.string_index[word] = in_str;
        if (F.colon) F.colon[word] = m.colon & ~in_str;
#pragma unroll
        for (int l = 0; l < LV; l++)
            if (l < p.num_levels) F.leveled[F.level_size * l + word] = lv[l];
    }
}

// The long tail of a line that runs past the slot: first '\n' from `from`
// (warp 0 of the index group); flags lines beyond max_ext past the tile.
__device__ int64_t find_line_end(const TileFile& p, int64_t from, int64_t tile_end, int64_t max_ext) {
    const int lane = threadIdx.x & 31;
    // four independent 16-byte loads per lane per step: 2 KiB per round
    // trip (a line of a megabyte is 512 steps; eight loads measured no
    // faster and cost the tile kernel registers); only bytes below `limit`
    // are read, those past it may still be on their way from the host
    constexpr int kChunks = 4;
    int64_t found = kNone;
    int64_t limit = p.n - tile_end > max_ext ? tile_end + max_ext : p.n;
    if (limit > p.avail) limit = p.avail;
    for (int64_t base = from; base < limit && found == kNone; base += 512 * kChunks) {
        uint4 v[kChunks];
#pragma unroll
        for (int c = 0; c < kChunks; c++) {
            const int64_t q = base + 512 * c + 16 * lane;
            v[c] = q + 16 <= limit ? __ldg(reinterpret_cast<const uint4*>(p.file + q)) : make_uint4(0, 0, 0, 0);
        }
        int64_t best = kNone;
#pragma unroll
        for (int c = kChunks - 1; c >= 0; c--) {  // the lowest chunk with a '\n' wins
            const int64_t q = base + 512 * c + 16 * lane;
            uint64_t nlbits = 0;
            if (q + 16 <= limit) {
                const uint32_t w4[4] = {v[c].x, v[c].y, v[c].z, v[c].w};
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    uint32_t f = eq_bytes(w4[i], 0x0A0A0A0Au);
                    while (f) {
                        nlbits |= 1ull << (4 * i + ((__ffs(f) - 1) >> 3));
                        f &= f - 1;
                    }
                }
            } else {
                for (int64_t j = q; j < limit; j++)
                    if (p.file[j] == '\n') nlbits |= 1ull << (j - q);
            }
            if (nlbits) best = q + ctz64(nlbits);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const int64_t o = __shfl_xor_sync(~0u, best, off);
            best = o < best ? o : best;
        }
        found = best;
    }
    if (found == kNone && limit < p.n) {
        if (lane == 0) atomicOr(p.status + 1, kErrLongLine);  // leave the input to the exact kernel
        return from;
    }
    return found == kNone ? p.n : found;
}

// The file of (batch-wide) tile t.
__device__ __forceinline__ void fetch_tile_file(const IndexParams& p, int64_t t, TileFile* out) {
    if (p.batch_files == 0) {
        *out = TileFile{p.file,     p.n,     p.avail,        p.string_index, p.leveled,
                        p.level_size, p.newline_bits, p.status, 0, p.colon};
        return;
    }
    int lo = 0, hi = p.batch_files - 1;  // last file with tile_begin <= t
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.batch[mid].tile_begin <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    *out = p.batch[lo];
}

// Starts the TMA copy of tile t into byte slot `slot` (one thread); the
// tile's file goes into sh.desc[dslot] before the copy's mbarrier arrive, so
// the threads that wait for the copy also see it.
template <class Sh>
__device__ __forceinline__ void start_tile(const IndexParams& p, Sh& sh, int64_t t, int slot, int dslot) {
    TileFile& F = sh.desc[dslot];
    fetch_tile_file(p, t, &F);
    const int64_t start = (t - F.tile_begin) * kTile;
    load_slot(F.file, start, F.avail - start < kSlotBytes ? F.avail - start : kSlotBytes, sh.bytes[slot],
              &sh.full[slot]);
}

// ---- index warps -------------------------------------------------------------
// The line kernel's warps 0-7: the tile's masks into a mask slot for the
// line warps that run beside them (newline index by look-back, in-kernel
// queries), and the index to device memory.
template <int LV>
__device__ void index_warps(const IndexParams& p, FShared<LV>& sh) {
    const int tid = threadIdx.x;  // 0..255
    unsigned long long* nl_agg = p.tile_state;
    const int64_t first_tile = p.tile_begin + blockIdx.x, stride = gridDim.x;
    if (tid == 0 && first_tile < p.tile_end) start_tile(p, sh, first_tile, 0, 0);
    int64_t k = 0;
    for (int64_t t = first_tile; t < p.tile_end; t += stride, ++k) {
        constexpr int kSlots = FShared<LV>::kByteSlots;
        const int bs = static_cast<int>(k % kSlots), ds = static_cast<int>(k % kRing), ms = static_cast<int>(k & 1);
        const uint32_t buse = static_cast<uint32_t>(k / kSlots), muse = static_cast<uint32_t>(k >> 1);
        // start the copy of the next tile: its byte slot was last used kSlots
        // tiles ago, once the line warps are done with its bytes
        if (tid == 0 && t + stride < p.tile_end) {
            const int nb = static_cast<int>((k + 1) % kSlots);
            const uint32_t nuse = static_cast<uint32_t>((k + 1) / kSlots);
            if (nuse > 0 && !mbar_wait_idle(&sh.bfree[nb], (nuse - 1) & 1)) atomicOr(p.status + 1, kErrCopyTimeout);
            start_tile(p, sh, t + stride, nb, static_cast<int>((k + 1) % kRing));
        }
        if (!mbar_wait_bounded(&sh.full[bs], buse & 1) && tid == 0) atomicOr(p.status + 1, kErrCopyTimeout);
        const uint8_t* buf = sh.bytes[bs];
        const TileFile& F = sh.desc[ds];
        const int64_t lt = t - F.tile_begin;  // the tile's index in its file

        const int64_t tile_start = lt * kTile;
        const int64_t tile_end = F.n - tile_start < kTile ? F.n : tile_start + kTile;
        const int64_t loaded_end = F.avail - tile_start < kSlotBytes ? F.avail : tile_start + kSlotBytes;
        const int64_t ws = tile_start + 64 * tid;

        // ---- one round over the slot: the tile's words and the look-ahead after it
        // One scan gives the tile's line starts, newline counts and every
        // word's state; the look-ahead words finish the tile's last line.
        const bool ahead = tid >= kTileWords;  // a word past the tile end
        const int slot = tid;                  // masks kept in shared memory for the line warps
        const uint64_t valid = bits_between(0, (ahead ? loaded_end : tile_end) - ws);
        ClassMasks m = load_classify(buf, tid);
        if (valid != ~0ull) restrict_masks(m, valid);
        // Escapes: a backslash run never crosses a '\n', so for every byte at
        // or after the tile's first line start the run found inside the slot
        // is the whole run (floor 0, parity 0 is exact there).
        uint32_t cout = 0;
        uint64_t esc;
        if (__any_sync(~0u, m.backslash != 0)) {
            const uint32_t cin = escape_carry_in(buf, tid, m.backslash, 0, 0);
            esc = escaped_mask(m.backslash, cin, &cout);
        } else {
            // no backslash in the warp's words: only the first byte of its
            // first word can be escaped, by a run ending just before it
            esc = (tid & 31) == 0 ? escape_scan_back(buf, tid, 0, 0) : 0u;
        }
        const uint64_t quotes = m.quote & ~esc;
        const uint64_t p0 = prefix_xor(quotes);
        const bool has_nl = m.newline != 0;
        const int f = has_nl ? ctz64(m.newline) : 0;
        const uint64_t after = has_nl ? (f == 63 ? 0ull : (~0ull << (f + 1))) : ~0ull;
        // in-string bits past the first '\n' when a line starts there
        const uint64_t pa = (p0 ^ (((p0 >> f) & 1ull) ? ~0ull : 0ull)) & after;
        const bool reset_w = has_nl && !ahead;  // only the tile's own newlines start lines here
        int q_w, d_abs = 0, dout_w = 0, din_w = 0;
        // quote parities from the prefix XOR: p0's bit 63 covers the word, bit f the bytes up to the '\n'
        const int par_all = static_cast<int>(p0 >> 63);
        if (reset_w) {
            q_w = par_all ^ static_cast<int>((p0 >> f) & 1ull);
            d_abs = -1 + popc64(m.open & after & ~pa) - popc64(m.close & after & ~pa);
        } else {
            q_w = par_all;
            dout_w = popc64(m.open & ~p0) - popc64(m.close & ~p0);
            din_w = popc64(m.open) - popc64(m.close) - dout_w;
        }
        // newlines of the tile count in the low 16 bits, of the look-ahead above
        const int nl_w = ahead ? (popc64(m.newline) << 16) : popc64(m.newline);
        if (tid == kIndexThreads - 1) sh.carry_esc = static_cast<int>(cout);
        // the file's first line starts at byte 0
        const TileScan sc = tile_scan(reset_w, q_w, d_abs, dout_w, din_w, nl_w, lt == 0, sh.rscan[k & 1]);
        const int tile_nl = sc.nl_total & 0xFFFF;
        const int ahead_nl = sc.nl_total >> 16;
        const bool lines_here = sc.lines_here != 0;  // a line starts in this tile
        if (tid == 0) st_release(nl_agg + t, tag48(p.epoch, static_cast<unsigned long long>(tile_nl)));
        // the mask slot was last used two tiles ago
        if (muse > 0 && !mbar_wait_idle(&sh.mfree[ms], (muse - 1) & 1) && tid == 0)
            atomicOr(p.status + 1, kErrCopyTimeout);
        // What this CTA finishes of the word, from which state; the branches
        // only choose it, so that finish_word runs converged below.
        bool act = false, own = true;
        ClassMasks wm = m;
        uint64_t wp0 = p0, check = 0;
        int ws_in = sc.s;
        int64_t wd_in = sc.d;
        if (!ahead) {
            const int excl = sc.nl_before & 0xFFFF;
            sh.nlmask[ms][tid] = m.newline;
            sh.nlexcl[ms][tid] = excl;
            uint64_t nm = m.newline;
            int q = excl;
            while (nm && q < kMaxTileLines) {
                sh.nlpos[ms][q++] = 64 * tid + ctz64(nm);
                nm &= nm - 1;
            }
            if (sc.reset) {
                // every byte of the word belongs to lines that start in this tile
                act = ws < tile_end;
                check = m.newline;
            } else if (has_nl) {
                // the tile's first line starts at byte f of this word
                sh.first_line = ws + f;
                restrict_masks(wm, after);
                act = true;
                own = f == 0;
                wp0 = pa;
                ws_in = 0;
                wd_in = -1;
                check = m.newline & after;
            }
        } else if (lines_here && (sc.nl_before >> 16) == 0 && valid) {
            // No '\n' between the tile end and this word: the tile's last line
            // runs into it.  The line ends at this word's first '\n' (the only
            // one checked here); a word that starts with it belongs to the next tile.
            if (has_nl) sh.ext_b = ws + f;
            act = !(has_nl && f == 0);
            check = has_nl ? (1ull << f) : 0ull;
        }
        finish_word<LV, true>(p, F, sh, ms, wm, wp0, ws_in, wd_in, ws >> 6, own, slot, valid, check, act);
        group_sync(kBarIndex, kIndexThreads);  // the tile's masks are complete in the slot

        const int64_t a_t = lt == 0 ? 0 : (lines_here ? sh.first_line : kNone);
        int64_t b_t = tile_end, hi = tile_end;
        if (lines_here && tile_end < F.n) {
            if (ahead_nl > 0) {
                b_t = sh.ext_b;
                hi = b_t;
            } else if (loaded_end == F.n) {
                b_t = F.n;
                hi = F.n;
            } else {
                // a line longer than the look-ahead: continue past the slot
                // straight from device memory
                const int s_in = sc.s_end;
                const int64_t d_in = sc.d_end;
                const int esc_in = sh.carry_esc;
                if (tid < 32) {
                    const int64_t e2 =
                        find_line_end(F, loaded_end, tile_end, p.max_extension > 0 ? p.max_extension : kMaxExtension);
                    if (tid == 0) sh.long_b = e2;
                }
                group_sync(kBarIndex, kIndexThreads);
                b_t = sh.long_b;
                hi = loaded_end;
                const int64_t own_end = (b_t + 63) & ~static_cast<int64_t>(63);
                int s = s_in, esc = esc_in;
                int64_t d = d_in;
                for (int64_t cs = loaded_end; cs < own_end && cs < F.n; cs += kRoundBytes) {
                    const int64_t cw = cs + 64 * tid;
                    const uint64_t cvalid = cw < own_end ? bits_between(0, F.n - cw) : 0ull;
                    ClassMasks c{0, 0, 0, 0, 0, 0, 0};
                    if (cvalid) {
                        c = classify_global(F.file, F.n, cw);
                        restrict_masks(c, cvalid);
                    }
                    // escape carry: previous word's trailing run, else the bytes before
                    const bool all_bs = c.backslash == ~0ull;
                    const int trail_par = all_bs ? 0 : (clz64(~c.backslash) & 1);
                    const int prev_par = __shfl_up_sync(~0u, trail_par, 1);
                    const int prev_all = __shfl_up_sync(~0u, all_bs ? 1 : 0, 1);
                    uint32_t ccin;
                    if ((tid & 31) > 0 && !prev_all) {
                        ccin = static_cast<uint32_t>(prev_par);
                    } else if (!cvalid) {
                        ccin = 0;  // a word past the line's end: never scan bytes past the file
                    } else {
                        int run = 0;
                        int64_t j = cw - 1;
                        while (j >= cs && __ldg(F.file + j) == '\\') {
                            ++run;
                            --j;
                        }
                        ccin = static_cast<uint32_t>((run & 1) ^ (j < cs ? esc : 0));
                    }
                    uint32_t ccout;
                    const uint64_t cesc = escaped_mask(c.backslash, ccin, &ccout);
                    const uint64_t cq = c.quote & ~cesc;
                    const uint64_t cp0 = prefix_xor(cq);
                    const Span csp{popc64(cq) & 1, popc64(c.open & ~cp0) - popc64(c.close & ~cp0),
                                   popc64(c.open) - popc64(c.close), 0};
                    Span ctotal;
                    const Span cex = index_scan_span(csp, sh.span_scratch, &ctotal);
                    const uint64_t ccheck =
                        (b_t >= cw && b_t < cw + 64) ? (c.newline & (1ull << (b_t - cw))) : 0ull;
                    finish_word<LV, true>(p, F, sh, ms, c, cp0, s ^ cex.q, d + (s ? (cex.ddt - cex.dd0) : cex.dd0),
                                          cw >> 6, true, -1, cvalid, ccheck, cvalid != 0);
                    if (tid == kIndexThreads - 1) sh.carry_esc = static_cast<int>(ccout);
                    group_sync(kBarIndex, kIndexThreads);
                    esc = sh.carry_esc;
                    d += s ? (ctotal.ddt - ctotal.dd0) : ctotal.dd0;
                    s ^= ctotal.q;
                    group_sync(kBarIndex, kIndexThreads);
                }
            }
        }
        if (tid == 0) {
            SlotInfo& in = sh.info[ms];
            in.a = a_t;
            in.b = b_t;
            in.hi = hi;
            in.tile_nl = tile_nl;
            in.byte_slot = bs;
            mbar_arrive(&sh.mready[ms]);  // the masks were complete at the barrier above
        }
    }
}

// ---- line warps --------------------------------------------------------------
template <int LV>
__device__ void line_warps(const IndexParams& p, FShared<LV>& sh) {
    const int lt = threadIdx.x - kIndexThreads;  // 0..127
    unsigned long long* nl_agg = p.tile_state;
    unsigned long long* nl_inc = p.tile_state + p.ntiles;
    // the queries' bytecode, from shared memory when it fits
    const bool ir_local = p.num_queries > 0 && p.num_queries <= kIrQueries && p.bytecode_bytes <= kIrBytes;
    if (ir_local) {
        for (int i = lt; i < p.bytecode_bytes; i += kLineThreads) sh.ir[i] = p.bytecode[i];
        for (int i = lt; i < p.num_queries; i += kLineThreads) sh.ir_off[i] = p.offsets[i];
        group_sync(kBarLines, kLineThreads);
    }
    const uint8_t* ir_base = ir_local ? sh.ir : p.bytecode;
    const int32_t* ir_off = ir_local ? sh.ir_off : p.offsets;
    int64_t k = 0;
    for (int64_t t = p.tile_begin + blockIdx.x; t < p.tile_end; t += gridDim.x, ++k) {
        const int ms = static_cast<int>(k & 1);
        const uint32_t muse = static_cast<uint32_t>(k >> 1);
        if (!mbar_wait_idle(&sh.mready[ms], muse & 1) && lt == 0) atomicOr(p.status + 1, kErrCopyTimeout);
        const SlotInfo in = sh.info[ms];
        const int64_t tile_start = t * kTile;
        if (lt < 32) {
            const int64_t before = lookback_newlines(nl_agg, nl_inc, t, in.tile_nl, p.epoch, p.status);
            if (lt == 0) {
                sh.nl_before = before;
                if (t == p.ntiles - 1) p.status[0] = static_cast<unsigned long long>(before + in.tile_nl + 1);
                if (t == 0 && p.newline_cap > 0 && p.materialize) p.newlines[0] = 0;
            }
        }
        group_sync(kBarLines, kLineThreads);
        const int64_t nl_before = sh.nl_before;
        if (p.materialize) {
            for (int w = lt; w < kTileWords; w += kLineThreads) {
                uint64_t nm = sh.nlmask[ms][w];
                int64_t idx = 1 + nl_before + sh.nlexcl[ms][w];
                while (nm) {
                    const int bit = ctz64(nm);
                    if (idx < p.newline_cap) p.newlines[idx] = tile_start + 64 * w + bit;
                    ++idx;
                    nm &= nm - 1;
                }
            }
        }
        if (p.num_queries > 0 && in.a != kNone) {
            if (in.tile_nl > kMaxTileLines) {
                if (lt == 0) atomicOr(p.status + 1, kErrDeferred);
            } else {
                const uint8_t* bytes = sh.bytes[in.byte_slot];
                LineView view{bytes - tile_start, p.n, sh.str[ms] - (tile_start >> 6),
                              &sh.lv[ms][0][0] - (tile_start >> 6), kSlotWords, in.hi,
                              sh.colon[ms] - (tile_start >> 6)};
                const int lines = in.tile_nl + (t == 0 ? 1 : 0);
                // a warp runs one query on up to 32 lines, so its lanes follow
                // the same opcode sequence
                const int chunks = (lines + 31) >> 5;
                const int tasks = chunks * p.num_queries;
                const int64_t per_line = 2 * static_cast<int64_t>(p.slots);
                const int32_t* nlpos = sh.nlpos[ms];
                for (int task = lt >> 5; task < tasks; task += kLineThreads / 32) {
                    const int q = task / chunks;
                    const int li = ((task - q * chunks) << 5) + (lt & 31);
                    if (li >= lines) continue;
                    int64_t start, line;
                    if (t == 0) {
                        start = li == 0 ? 0 : tile_start + nlpos[li - 1];
                        line = li;
                    } else {
                        start = tile_start + nlpos[li];
                        line = 1 + nl_before + li;
                    }
                    const int nxt = t == 0 ? li : li + 1;
                    const int64_t end = nxt < in.tile_nl ? tile_start + nlpos[nxt] : in.b;
                    if (line >= p.out_lines) {
                        atomicOr(p.status + 1, kErrOutOverflow);
                        continue;
                    }
                    int64_t* res = p.out + (static_cast<int64_t>(q) * p.out_lines + line) * per_line;
                    for (int64_t r = 0; r < per_line; r++) res[r] = -1;
                    PackedLevels lv{&sh.lvl_end[0][lt], &sh.lvl_idx[0][lt], kLineThreads, LV + 1, start};
                    if (end > in.hi ||
                        run_line_with(view, start, end, ir_base + ir_off[q], res, lv) == kLineDeferred)
                        atomicOr(p.status + 1, kErrDeferred);
                }
            }
        }
        group_sync(kBarLines, kLineThreads);
        if (lt == 0) {
            mbar_arrive(&sh.mfree[ms]);
            mbar_arrive(&sh.bfree[in.byte_slot]);
        }
    }
}

template <int LV>
__global__ void __launch_bounds__(kThreads, 2) line_index_kernel(IndexParams p) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    FShared<LV>& sh = *reinterpret_cast<FShared<LV>*>(smem_raw);
    if (threadIdx.x == 0) {
        for (int i = 0; i < kRing; i++) {
            mbar_init(&sh.full[i], 1);
            mbar_init(&sh.bfree[i], 1);
        }
        for (int i = 0; i < kMaskSlots; i++) {
            mbar_init(&sh.mready[i], 1);
            mbar_init(&sh.mfree[i], 1);
        }
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x < kIndexThreads)
        index_warps<LV>(p, sh);
    else
        line_warps<LV>(p, sh);
}

// ---- standalone index kernel ---------------------------------------------
// Index builds without in-kernel queries (the default): 128 threads, each
// owning four consecutive 64-byte words (256 bytes) of a 32 KiB slot, which
// holds a 30 KiB tile and its 2 KiB look-ahead.  A thread classifies its
// words one after another and composes their effect on the scan state
// (string state, level, newline count) itself, so the warp scan, the
// cross-warp scan and the tile's bookkeeping are paid once per four words.
// What a word's classification leaves for the second pass (its masks and
// level changes) is kept in shared memory where the word's bytes were, so
// the slot holds bytes, then masks, then the level split's inputs and (up
// to four levels) the level masks, and six CTAs fit per SM.  The level split deals the warp's words that hold
// bracket cuts over its lanes (deal_levels).  Writes the string index, the ':'
// bitmap, the leveled bitmaps and the '\n' bitmap with one 32-byte store per
// thread and bitmap where all four words are its own, and every tile's
// newline count; no tile waits for another.  Ownership of words and lines
// is the line kernel's (see the top of this file), with tiles of
// kStandaloneTileBytes.
constexpr int kWThreads = 128;
constexpr int kWWarps = kWThreads / 32;
constexpr int kWK = 4;                                     // consecutive words per thread
constexpr int kWLaneBytes = 64 * kWK;                      // 256
constexpr int64_t kWSlot = kWThreads * kWLaneBytes;        // 32 KiB
constexpr int64_t kWTile = kStandaloneTileBytes;           // 30 KiB
constexpr int kWTileLanes = static_cast<int>(kWTile / kWLaneBytes);  // threads 0..119: the tile
constexpr int kWSlotWords = static_cast<int>(kWSlot / 64);           // 512
constexpr int64_t kWRound = kWThreads * 64;                // extension rounds: one word per thread
static_assert(kWTile % kWLaneBytes == 0 && kWSlot - kWTile == kExtBytes, "tile + 2 KiB look-ahead per slot");

// With at most four levels a word's level masks go into cells 0-3 of the
// word itself (word_cell) once the level split has read them; with more
// they need an array of their own, which lowers the CTAs per SM.
template <int LV>
constexpr bool kCellLevels = LV <= 4;

template <int LV>
struct WShared {
    // the tile's bytes (TMA destination); after a word is classified, its
    // 64 bytes hold eight 8-byte cells of its state (word_cell)
    uint8_t bytes[kWSlot];
    union {
        // level masks, at i * kWThreads + thread (deal_levels); unused with kCellLevels
        uint64_t acc[kCellLevels<LV> ? 1 : LV][kCellLevels<LV> ? 1 : kWSlotWords];
        uint64_t lvacc[kWWarps][LV][32];  // split_levels_warp in the extension rounds
    };
    TileFile desc[2];  // the file of tile k in desc[k & 1]
    uint64_t full;     // the slot's TMA barrier (phase k & 1 for tile k)
    Span span_scratch[kWWarps];
    WarpSum rscan[2][kWWarps];
    int carry_esc;
    int64_t long_b;
    int64_t next_tile;  // the tile claimed for the next round
};

// Cell c (0..7) of word i of thread g, in the bytes the word was loaded
// into.  Cells are rotated by the thread so that the threads of a warp
// spread over the banks.  First pass: 0 quote prefix XOR, 1 '{['
// (outside strings or not), 2 '}]', 3 structural, 4 ':', 5 '\n', 6 level
// changes entered outside / inside a string, 7 quote parity or the string
// state after a reset.  Second pass: 0 opening brackets, 1 closing
// brackets, 2 structural bytes, 3 level at the word's first byte, all of
// the word's own and outside strings; 4 string mask, 5 '\n' as before,
// 6 ':' outside strings.  With kCellLevels, cells 0-3 then hold the masks
// of levels 0-3: written in the second pass for a word without bracket
// cuts, by deal_levels for a word with some.
__device__ __forceinline__ uint64_t* word_cell(uint8_t* slot, int g, int i, int c) {
    return reinterpret_cast<uint64_t*>(slot + kWLaneBytes * g + 64 * i + 8 * ((c + g) & 7));
}

// One 32-byte store of four words where all four are to be written and the
// destination is 32-byte aligned, else one store per word of `mask`.
__device__ __forceinline__ void store_words4(uint64_t* dst, const uint64_t (&v)[4], unsigned mask) {
    if (mask == 0xFu && (reinterpret_cast<uintptr_t>(dst) & 31) == 0) {
        asm volatile("st.global.v4.b64 [%0], {%1, %2, %3, %4};" ::"l"(dst), "l"(v[0]), "l"(v[1]), "l"(v[2]),
                     "l"(v[3])
                     : "memory");
    } else {
#pragma unroll
        for (int i = 0; i < 4; i++)
            if ((mask >> i) & 1u) dst[i] = v[i];
    }
}

// Starts the TMA copy of tile t into the slot (one thread); its file goes
// into desc[dslot] before the copy's arrive.
template <int LV>
__device__ __forceinline__ void start_wide_tile(const IndexParams& p, WShared<LV>& sh, int64_t t, int dslot) {
    TileFile& F = sh.desc[dslot];
    fetch_tile_file(p, t, &F);
    const int64_t start = (t - F.tile_begin) * kWTile;
    load_slot(F.file, start, F.avail - start < kWSlot ? F.avail - start : kWSlot, sh.bytes, &sh.full);
}

// The level split of the warp's words that hold bracket cuts (inputs in
// cells 0-3 of each word; the other words' level masks are already in
// place, sh.acc or their cells 0-3): such words are dealt out over the 32 lanes, one per lane per
// pass, and each is split by split_levels, which walks its cuts.  A
// quarter of the words have cuts and their counts differ a lot (tweets: 0.87
// per word on average, many with eight or more), so dealing them over the
// warp keeps most lanes busy, where a loop per thread would run as long as
// the warp's densest thread.  `cmask`: which of the thread's four words have
// cuts.
template <int LV>
__device__ __forceinline__ void deal_levels(WShared<LV>& sh, unsigned cmask) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m = __popc(cmask);
    int incl = m;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int o = __shfl_up_sync(~0u, incl, off);
        if (lane >= off) incl += o;
    }
    const int base = incl - m;
    const int total = __shfl_sync(~0u, incl, 31);
    __syncwarp();
    for (int r = 0; r < total; r += 32) {
        const int g = r + lane;  // this lane's word with cuts, numbered across the warp
        int o = 0;               // its thread: the last lane whose first number is <= g
#pragma unroll
        for (int s = 16; s > 0; s >>= 1)
            if (__shfl_sync(~0u, base, o + s) <= g) o += s;
        const unsigned cm = __shfl_sync(~0u, cmask, o);
        int c = g - __shfl_sync(~0u, base, o);  // number within thread o
        int wi = 0;                              // its word: the c-th set bit of cm
#pragma unroll
        for (int b = 0; b < kWK; b++) {
            const int has = (cm >> b) & 1u;
            if (has && c == 0) wi = b;
            c -= has;
        }
        if (g < total) {
            const int og = 32 * warp + o;
            const uint64_t op = *word_cell(sh.bytes, og, wi, 0), cl = *word_cell(sh.bytes, og, wi, 1);
            const uint64_t st = *word_cell(sh.bytes, og, wi, 2);
            const int dd = static_cast<int>(static_cast<int64_t>(*word_cell(sh.bytes, og, wi, 3)));
            uint64_t lv[LV];
            split_levels<LV>(op, cl, st, dd, lv);
#pragma unroll
            for (int l = 0; l < LV; l++) {
                if constexpr (kCellLevels<LV>)
                    *word_cell(sh.bytes, og, wi, l) = lv[l];
                else
                    sh.acc[l][wi * kWThreads + og] = lv[l];
            }
        }
    }
    __syncwarp();
}

// A line that runs past the slot: the rest of it, up to its '\n', from
// device memory, one word per thread per round (the line kernel's long-line
// path with 128 threads).  s_in / d_in: the scan state after the slot.
template <int LV>
__device__ void extend_long_line(const IndexParams& p, const TileFile& F, WShared<LV>& sh, int64_t loaded_end,
                                 int64_t tile_end, int s_in, int64_t d_in) {
    const int tid = threadIdx.x;
    if (tid < 32) {
        const int64_t e2 =
            find_line_end(F, loaded_end, tile_end, p.max_extension > 0 ? p.max_extension : kMaxExtension);
        if (tid == 0) {
            sh.long_b = e2;
            // the escape state at loaded_end: the backslash run before it
            // lies in the line, which starts in this tile with a '\n'
            int run = 0;
            for (int64_t j = loaded_end - 1; j >= 0 && F.file[j] == '\\'; --j) ++run;
            sh.carry_esc = run & 1;
        }
    }
    group_sync(kBarIndex, kWThreads);
    const int64_t b_t = sh.long_b;
    const int64_t own_end = (b_t + 63) & ~static_cast<int64_t>(63);
    int s = s_in, esc = sh.carry_esc;
    int64_t d = d_in;
    for (int64_t cs = loaded_end; cs < own_end && cs < F.n; cs += kWRound) {
        const int64_t cw = cs + 64 * tid;
        const uint64_t cvalid = cw < own_end ? bits_between(0, F.n - cw) : 0ull;
        ClassMasks c{0, 0, 0, 0, 0, 0, 0};
        if (cvalid) {
            c = classify_global(F.file, F.n, cw);
            restrict_masks(c, cvalid);
        }
        // escape carry: previous word's trailing run, else the bytes before
        const bool all_bs = c.backslash == ~0ull;
        const int trail_par = all_bs ? 0 : (clz64(~c.backslash) & 1);
        const int prev_par = __shfl_up_sync(~0u, trail_par, 1);
        const int prev_all = __shfl_up_sync(~0u, all_bs ? 1 : 0, 1);
        uint32_t ccin;
        if ((tid & 31) > 0 && !prev_all) {
            ccin = static_cast<uint32_t>(prev_par);
        } else if (!cvalid) {
            ccin = 0;  // a word past the line's end: never scan bytes past the file
        } else {
            int run = 0;
            int64_t j = cw - 1;
            while (j >= cs && __ldg(F.file + j) == '\\') {
                ++run;
                --j;
            }
            ccin = static_cast<uint32_t>((run & 1) ^ (j < cs ? esc : 0));
        }
        uint32_t ccout;
        const uint64_t cesc = escaped_mask(c.backslash, ccin, &ccout);
        const uint64_t cq = c.quote & ~cesc;
        const uint64_t cp0 = prefix_xor(cq);
        const Span csp{popc64(cq) & 1, popc64(c.open & ~cp0) - popc64(c.close & ~cp0), popc64(c.open) - popc64(c.close),
                       0};
        Span ctotal;
        const Span cex = index_scan_span<kWWarps>(csp, sh.span_scratch, &ctotal);
        const uint64_t ccheck = (b_t >= cw && b_t < cw + 64) ? (c.newline & (1ull << (b_t - cw))) : 0ull;
        finish_word<LV, false>(p, F, sh, 0, c, cp0, s ^ cex.q, d + (s ? (cex.ddt - cex.dd0) : cex.dd0), cw >> 6, true,
                               -1, cvalid, ccheck, cvalid != 0);
        if (tid == kWThreads - 1) sh.carry_esc = static_cast<int>(ccout);
        group_sync(kBarIndex, kWThreads);
        esc = sh.carry_esc;
        d += s ? (ctotal.ddt - ctotal.dd0) : ctotal.dd0;
        s ^= ctotal.q;
        group_sync(kBarIndex, kWThreads);
    }
}

// Up to four levels: 6 CTAs per SM (about 37 KiB of shared memory each,
// at most 85 registers a thread); more levels add the level-mask array.
template <int LV>
__global__ void __launch_bounds__(kWThreads, LV <= 4 ? 6 : (LV <= 8 ? 3 : 2)) tile_index_kernel(IndexParams p) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    WShared<LV>& sh = *reinterpret_cast<WShared<LV>*>(smem_raw);
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&sh.full, 1);
        fence_mbar_init();
    }
    // Tiles are pulled one at a time from p.tile_counter (zeroed before the
    // launch), so a CTA that follows a long line past its tile takes fewer
    // of them; a tile never waits for another, so any claim order is safe.
    if (tid == 0) {
        const int64_t t0 = p.tile_begin + static_cast<int64_t>(atomicAdd(p.tile_counter, 1u));
        sh.next_tile = t0;
        if (t0 < p.tile_end) start_wide_tile(p, sh, t0, 0);
    }
    __syncthreads();
    int64_t k = 0;
    for (int64_t t = sh.next_tile; t < p.tile_end; ++k) {
        if (!mbar_wait_bounded(&sh.full, static_cast<uint32_t>(k & 1)) && tid == 0)
            atomicOr(p.status + 1, kErrCopyTimeout);
        uint8_t* slot = sh.bytes;
        const TileFile& F = sh.desc[k & 1];
        const int64_t lt = t - F.tile_begin;  // the tile's index in its file
        const int64_t tile_start = lt * kWTile;
        const int64_t tile_end = F.n - tile_start < kWTile ? F.n : tile_start + kWTile;
        const int64_t loaded_end = F.avail - tile_start < kWSlot ? F.avail : tile_start + kWSlot;
        const bool ahead = tid >= kWTileLanes;  // the thread's words lie in the look-ahead
        const int64_t lane_start = tile_start + kWLaneBytes * tid;
        const int64_t vend = ahead ? loaded_end : tile_end;

        // ---- first pass: classify the thread's four words, compose their scan effect
        // The escape state entering the thread's bytes: a backslash run never
        // crosses a '\n', so inside the slot the run before them is the whole
        // run.  Read before any thread overwrites its bytes.
        uint32_t cin = escape_scan_back(slot, kWK * tid, 0, 0);
        group_sync(kBarIndex, kWThreads);
        int l_reset = 0, l_s = 0, l_dout = 0, l_din = 0, l_nl = 0;
#pragma unroll 1
        for (int i = 0; i < kWK; i++) {
            const int64_t ws = lane_start + 64 * i;
            const uint64_t valid = bits_between(0, vend - ws);
            // the thread's words are 256 bytes apart from the next thread's,
            // so a rotation by word would be the same for every thread
            ClassMasks m = load_classify<false>(slot, kWK * tid + i);
            if (valid != ~0ull) restrict_masks(m, valid);
            uint32_t cout = 0;
            const uint64_t esc = (m.backslash | cin) ? escaped_mask(m.backslash, cin, &cout) : 0ull;
            cin = cout;
            const uint64_t p0 = prefix_xor(m.quote & ~esc);
            const bool has_nl = m.newline != 0;
            const int f = has_nl ? ctz64(m.newline) : 0;
            const int par_all = static_cast<int>(p0 >> 63);
            int wq, wa, wb;
            if (has_nl && !ahead) {
                // a line starts after the word's first '\n': the state after the word is absolute
                const uint64_t after = f == 63 ? 0ull : (~0ull << (f + 1));
                const uint64_t pa = (p0 ^ (((p0 >> f) & 1ull) ? ~0ull : 0ull)) & after;
                wq = par_all ^ static_cast<int>((p0 >> f) & 1ull);
                wa = -1 + popc64(m.open & after & ~pa) - popc64(m.close & after & ~pa);
                wb = 0;
                l_reset = 1;
                l_s = wq;
                l_dout = wa;
            } else {
                wq = par_all;
                wa = popc64(m.open & ~p0) - popc64(m.close & ~p0);  // entered outside a string
                wb = popc64(m.open) - popc64(m.close) - wa;        // entered inside
                if (l_reset) {
                    l_dout += l_s ? wb : wa;
                } else {
                    const int a = l_dout + (l_s ? wb : wa);
                    l_din += l_s ? wa : wb;
                    l_dout = a;
                }
                l_s ^= wq;
            }
            l_nl += ahead ? (popc64(m.newline) << 16) : popc64(m.newline);
            *word_cell(slot, tid, i, 0) = p0;
            *word_cell(slot, tid, i, 1) = m.open;
            *word_cell(slot, tid, i, 2) = m.close;
            *word_cell(slot, tid, i, 3) = m.structural;
            *word_cell(slot, tid, i, 4) = m.colon;
            *word_cell(slot, tid, i, 5) = m.newline;
            *word_cell(slot, tid, i, 6) = static_cast<uint32_t>(wa) | (static_cast<uint64_t>(static_cast<uint32_t>(wb)) << 32);
            *word_cell(slot, tid, i, 7) = static_cast<uint64_t>(wq);
        }
        const TileScan sc = tile_scan<kWWarps, 64 * kWK>(l_reset != 0, l_s, l_dout, l_dout, l_din, l_nl, lt == 0,
                                                         sh.rscan[k & 1]);
        if (tid == 0) p.tile_newlines[t] = sc.nl_total & 0xFFFF;
        const int ahead_nl = sc.nl_total >> 16;
        const bool lines_here = sc.lines_here != 0;  // a line starts in this tile

        // ---- second pass: final masks of the four words from the state at each one's first byte
        int rb = sc.reset, s = sc.s, d = sc.d, nlb = sc.nl_before;
        unsigned wmask = 0, cmask = 0;
#pragma unroll 1
        for (int i = 0; i < kWK; i++) {
            const int64_t ws = lane_start + 64 * i;
            const uint64_t valid = bits_between(0, vend - ws);
            const uint64_t p0 = *word_cell(slot, tid, i, 0), wopen = *word_cell(slot, tid, i, 1);
            const uint64_t wclose = *word_cell(slot, tid, i, 2), wst = *word_cell(slot, tid, i, 3);
            const uint64_t wcolon = *word_cell(slot, tid, i, 4), nl = *word_cell(slot, tid, i, 5);
            const uint64_t ab = *word_cell(slot, tid, i, 6);
            const int wq = static_cast<int>(*word_cell(slot, tid, i, 7));
            const int wa = static_cast<int32_t>(static_cast<uint32_t>(ab)), wb = static_cast<int32_t>(ab >> 32);
            const bool has_nl = nl != 0;
            const int f = has_nl ? ctz64(nl) : 0;
            const uint64_t after = has_nl ? (f == 63 ? 0ull : (~0ull << (f + 1))) : ~0ull;
            // what this CTA finishes of the word, from which state
            bool act = false, own = true;
            uint64_t keep = ~0ull, wp0 = p0, check = 0;
            int s_in = s, d_in = d;
            if (!ahead) {
                if (rb) {
                    // every byte of the word belongs to lines that start in this tile
                    act = ws < tile_end;
                    check = nl;
                } else if (has_nl) {
                    // the tile's first line starts after byte f of this word
                    keep = after;
                    act = true;
                    own = f == 0;
                    wp0 = (p0 ^ (((p0 >> f) & 1ull) ? ~0ull : 0ull)) & after;
                    s_in = 0;
                    d_in = -1;
                    check = nl & after;
                }
            } else if (lines_here && (nlb >> 16) == 0 && valid) {
                // no '\n' between the tile end and this word: the tile's last
                // line runs into it and ends at its first '\n' (the only one checked)
                act = !(has_nl && f == 0);
                check = has_nl ? (1ull << f) : 0ull;
            }
            const uint64_t in_str = (wp0 ^ (s_in ? ~0ull : 0ull)) & valid;
            const uint64_t open = wopen & keep & ~in_str, close = wclose & keep & ~in_str;
            if (act && check) {
                // every checked '\n' must be outside strings at level -1
                if (check & in_str) atomicOr(F.status + 1, kErrIrregular);
                for (uint64_t c = check; c; c &= c - 1) {
                    const uint64_t below = (1ull << ctz64(c)) - 1;
                    if (d_in + popc64(open & below) - popc64(close & below) != -1) atomicOr(F.status + 1, kErrIrregular);
                }
            }
            const bool split = act && own;
            const uint64_t sk = split ? ~0ull : 0ull;
            const uint64_t op = open & sk, cl = close & sk, st = wst & keep & ~in_str & sk;
            const int dd = d_in > 128 ? 128 : (d_in < -128 ? -128 : d_in);
            const bool cut = (op | (cl << 1)) != 0;
            // a word without bracket cuts is all at its first level (words
            // with cuts are split by deal_levels)
            if (kCellLevels<LV> && !cut) {
#pragma unroll
                for (int l = 0; l < LV; l++) *word_cell(slot, tid, i, l) = dd == l ? st : 0ull;
            } else {
                *word_cell(slot, tid, i, 0) = op;
                *word_cell(slot, tid, i, 1) = cl;
                *word_cell(slot, tid, i, 2) = st;
                *word_cell(slot, tid, i, 3) = static_cast<uint64_t>(static_cast<int64_t>(dd));
                if constexpr (!kCellLevels<LV>) {
#pragma unroll
                    for (int l = 0; l < LV; l++) sh.acc[l][i * kWThreads + tid] = dd == l ? st : 0ull;
                }
            }
            *word_cell(slot, tid, i, 4) = in_str;
            *word_cell(slot, tid, i, 6) = wcolon & keep & ~in_str;
            cmask |= cut ? (1u << i) : 0u;
            wmask |= split ? (1u << i) : 0u;
            // the state at the next word's first byte
            if (has_nl && !ahead) {
                rb = 1;
                s = wq;
                d = wa;
            } else {
                d += s ? wb : wa;
                s ^= wq;
            }
            nlb += ahead ? (popc64(nl) << 16) : popc64(nl);
        }
        deal_levels<LV>(sh, cmask);
        // ---- the thread's words to the index
        if (!ahead) {  // the '\n' bitmap of the tile's words
            const unsigned own_nl =
                lane_start + kWLaneBytes <= tile_end
                    ? 0xFu
                    : (lane_start < tile_end ? ((1u << ((tile_end - lane_start + 63) >> 6)) - 1u) : 0u);
            if (own_nl) {
                uint64_t v[kWK];
#pragma unroll
                for (int i = 0; i < kWK; i++) v[i] = *word_cell(slot, tid, i, 5);
                store_words4(F.newline_bits + (lane_start >> 6), v, own_nl);
            }
        }
        if (p.materialize && wmask) {
            const int64_t w0 = lane_start >> 6;
            uint64_t v[kWK];
#pragma unroll
            for (int i = 0; i < kWK; i++) v[i] = *word_cell(slot, tid, i, 4);
            store_words4(F.string_index + w0, v, wmask);
            if (F.colon) {
#pragma unroll
                for (int i = 0; i < kWK; i++) v[i] = *word_cell(slot, tid, i, 6);
                store_words4(F.colon + w0, v, wmask);
            }
#pragma unroll
            for (int l = 0; l < LV; l++) {
                if (l < p.num_levels) {
#pragma unroll
                    for (int i = 0; i < kWK; i++) {
                        if constexpr (kCellLevels<LV>)
                            v[i] = *word_cell(slot, tid, i, l);
                        else
                            v[i] = sh.acc[l][i * kWThreads + tid];
                    }
                    store_words4(F.leveled + F.level_size * l + w0, v, wmask);
                }
            }
        }
        group_sync(kBarIndex, kWThreads);  // the slot and sh.acc are read: the next tile's copy may start
        // a line past the slot is finished before the next claim, so that
        // the tiles go to CTAs that are free
        if (lines_here && tile_end < F.n && ahead_nl == 0 && loaded_end < F.n)
            extend_long_line<LV>(p, F, sh, loaded_end, tile_end, sc.s_end, sc.d_end);
        if (tid == 0) {
            const int64_t nt = p.tile_begin + static_cast<int64_t>(atomicAdd(p.tile_counter, 1u));
            sh.next_tile = nt;
            if (nt < p.tile_end) start_wide_tile(p, sh, nt, static_cast<int>((k + 1) & 1));
        }
        group_sync(kBarIndex, kWThreads);  // the next tile's number is visible
        t = sh.next_tile;
    }
}

// Raises a kernel's dynamic shared memory limit, once per device (the
// attribute belongs to the kernel's instance on the current device).
template <class Kernel>
cudaError_t prepare(Kernel kernel, size_t smem, std::atomic<unsigned long long>& done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done.load() & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e == cudaSuccess && bit) done.fetch_or(bit);
    return e;
}

template <int LV, bool kLines>
struct KernelOf {
    static void* fn() {
        return kLines ? reinterpret_cast<void*>(line_index_kernel<LV>) : reinterpret_cast<void*>(tile_index_kernel<LV>);
    }
    static size_t smem() { return kLines ? sizeof(FShared<LV>) : sizeof(WShared<LV>); }
    static int threads() { return kLines ? kThreads : kWThreads; }
    static std::atomic<unsigned long long>& done() {
        static std::atomic<unsigned long long> d{0};
        return d;
    }
};

template <int LV, bool kLines>
int occupancy() {
    using K = KernelOf<LV, kLines>;
    if (prepare(K::fn(), K::smem(), K::done()) != cudaSuccess) return -1;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, K::fn(), K::threads(), K::smem()) != cudaSuccess)
        return -1;
    return blocks;
}

template <int LV, bool kLines>
cudaError_t launch(const IndexParams& p, int grid, cudaStream_t stream) {
    using K = KernelOf<LV, kLines>;
    cudaError_t e = prepare(K::fn(), K::smem(), K::done());
    if (e != cudaSuccess) return e;
    if (kLines)
        line_index_kernel<LV><<<grid, kThreads, sizeof(FShared<LV>), stream>>>(p);
    else
        tile_index_kernel<LV><<<grid, kWThreads, sizeof(WShared<LV>), stream>>>(p);
    return cudaGetLastError();
}

}  // namespace

int line_index_max_ctas_per_sm(int lv) {
    if (lv <= 4) return occupancy<4, true>();
    if (lv <= 8) return occupancy<8, true>();
    return occupancy<16, true>();
}

cudaError_t launch_line_index_kernel(const IndexParams& p, int grid, cudaStream_t stream) {
    if (p.num_levels <= 4) return launch<4, true>(p, grid, stream);
    if (p.num_levels <= 8) return launch<8, true>(p, grid, stream);
    return launch<16, true>(p, grid, stream);
}

int tile_index_max_ctas_per_sm(int lv) {
    if (lv <= 4) return occupancy<4, false>();
    if (lv <= 8) return occupancy<8, false>();
    return occupancy<16, false>();
}

cudaError_t launch_tile_index_kernel(const IndexParams& p, int grid, cudaStream_t stream) {
    if (p.num_levels <= 4) return launch<4, false>(p, grid, stream);
    if (p.num_levels <= 8) return launch<8, false>(p, grid, stream);
    return launch<16, false>(p, grid, stream);
}

}  // namespace gpj
