// Exact single-pass structural index on sm_100a (any input).
//
// Replaces the reference's seven index launches and three host round trips
// (stages/CombinedIndex.java:28-151, stages/LeveledBitmapsIndex.java:40-103,
// kernels create_combined_escape_carry_newline_count_index.cu,
// create_combined_escape_newline_index.cu, create_quote_index.cu,
// create_string_index.cu, create_leveled_bitmaps_carry_index.cu,
// create_leveled_bitmaps.cu) with one persistent kernel.  It is the fallback
// of the line-parallel kernel (index_lines.cu) for inputs that are not
// well-formed NDJSON:
//
//  * The input is cut into 16 KiB tiles claimed in order from an atomic
//    counter.  Each CTA (256 threads, one 64-byte word per thread) double
//    buffers its tiles in shared memory with 1-D TMA bulk copies.
//  * Each thread classifies its 64 bytes into bit masks (word_ops.cuh),
//    resolves escapes with a carry taken from the previous word (warp
//    shuffle) or, at the tile start, from the bytes before the tile.
//  * Word summaries (quote parity, depth change, newline count) are scanned
//    across the tile; the tile summary is published for a decoupled
//    look-back, which supplies the string state, level counter and newline
//    count before the tile (the carries the reference scans on the host).
//  * Each thread then writes its string-index word, its words of the
//    leveled bitmaps and its newline offsets: one tile later, from the
//    word's state kept in its own bytes of the tile buffer, while warp 0
//    looks back for the next tile (the look-back's wait overlaps the
//    stores of the tile before).
//
// Output layouts are the reference's: string_index u64[ceil(n/64)],
// leveled u64[num_levels][ceil(n/64)], newline index i64[lines] with [0]=0.
#include <cstdint>

#include "device_common.cuh"
#include "index_kernel.h"
#include "word_ops.cuh"

namespace gpj {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int64_t kTile = kIndexTileBytes;  // 256 threads x 64 bytes
static_assert(kTile == kThreads * 64, "one word per thread");

// Tile state words (3 per tile), each tagged with the launch epoch in its top
// 16 bits so the array never needs clearing between launches.
//   AGG : q(1) | nl(15) | dd0+16384 (16) | ddt+16384 (16)
//   INCA: s(1) | d + 2^46 (47)
//   INCB: nl (48)
constexpr unsigned long long kPayload48 = (1ull << 48) - 1;

__device__ __forceinline__ unsigned long long tag(uint32_t epoch, unsigned long long payload) {
    return (static_cast<unsigned long long>(epoch) << 48) | (payload & kPayload48);
}
__device__ __forceinline__ bool tagged(unsigned long long w, uint32_t epoch) {
    return static_cast<uint32_t>(w >> 48) == epoch;
}

__device__ __forceinline__ unsigned long long pack_agg(const Span& a) {
    return (static_cast<unsigned long long>(a.q & 1) << 47) |
           (static_cast<unsigned long long>(a.nl) << 32) |
           (static_cast<unsigned long long>(a.dd0 + 16384) << 16) |
           static_cast<unsigned long long>(a.ddt + 16384);
}
__device__ __forceinline__ Span unpack_agg(unsigned long long w) {
    Span a;
    a.q = static_cast<int32_t>((w >> 47) & 1);
    a.nl = static_cast<int32_t>((w >> 32) & 0x7FFF);
    a.dd0 = static_cast<int32_t>((w >> 16) & 0xFFFF) - 16384;
    a.ddt = static_cast<int32_t>(w & 0xFFFF) - 16384;
    return a;
}

// State before/after a tile.
struct Carry {
    int s;       // inside a string
    int64_t d;   // level counter
    int64_t nl;  // newlines so far
};

// Aggregate of a run of tiles with 64-bit counters (look-back accumulator).
struct Span64 {
    int q;
    int64_t dd0, ddt, nl;
};

__device__ __forceinline__ Span64 widen(const Span& a) { return Span64{a.q, a.dd0, a.ddt, a.nl}; }

__device__ __forceinline__ Span64 compose64(const Span64& a, const Span64& b) {
    return Span64{a.q ^ b.q, a.dd0 + (a.q ? b.ddt - b.dd0 : b.dd0), a.ddt + b.ddt, a.nl + b.nl};
}

__device__ __forceinline__ Carry apply(const Carry& c, const Span64& a) {
    return Carry{c.s ^ a.q, c.d + (c.s ? a.ddt - a.dd0 : a.dd0), c.nl + a.nl};
}

__device__ __forceinline__ Span shfl_span_up(const Span& v, int off) {
    return Span{__shfl_up_sync(~0u, v.q, off), __shfl_up_sync(~0u, v.dd0, off),
                __shfl_up_sync(~0u, v.ddt, off), __shfl_up_sync(~0u, v.nl, off)};
}

__device__ __forceinline__ Span64 shfl_span64_down(const Span64& v, int off) {
    return Span64{__shfl_down_sync(~0u, v.q, off), __shfl_down_sync(~0u, v.dd0, off),
                  __shfl_down_sync(~0u, v.ddt, off), __shfl_down_sync(~0u, v.nl, off)};
}

// Parity of the backslash run that ends just before byte `pos` (the escape
// state of byte `pos`), however long the run (Sequential.java:36-64 has no
// bound either).  `pos` is a tile start, a multiple of 16, so the bytes
// before it are read as aligned 16-byte vectors, four at a time.
__device__ int escape_parity_before(const uint8_t* file, int64_t pos) {
    int64_t run = 0;
    for (int64_t k = pos; k > 0; k -= 64) {
        const int64_t lo = k - 64 > 0 ? k - 64 : 0;
        uint4 q[4];
#pragma unroll
        for (int j = 0; j < 4; j++)  // the 16-byte vectors ending at k, k - 16, ...
            q[j] = k - 16 * (j + 1) >= lo ? __ldg(reinterpret_cast<const uint4*>(file + k - 16 * (j + 1)))
                                          : make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (k - 16 * (j + 1) < lo) return static_cast<int>(run & 1);  // the file's first byte
            const uint32_t w[4] = {q[j].w, q[j].z, q[j].y, q[j].x};  // highest bytes first
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t nb = ~eq_bytes(w[i], 0x5C5C5C5Cu) & 0x80808080u;  // non-backslash bytes
                if (nb) return static_cast<int>((run + (__clz(nb) >> 3)) & 1);
                run += 4;
            }
        }
    }
    return static_cast<int>(run & 1);
}

// Look-back: state before tile t, given its aggregate.  Executed by one
// warp; publishes the tile's inclusive state before returning.
__device__ Carry look_back(unsigned long long* states, int64_t t, const Span& agg, uint32_t epoch,
                           unsigned long long* status) {
    const int lane = threadIdx.x & 31;
    Carry before{0, -1, 0};
    if (t > 0) {
        if (lane == 0) st_release(states + 3 * t, tag(epoch, pack_agg(agg)));
        Span64 acc{0, 0, 0, 0};
        int64_t base = t - 1;
        unsigned polls = 0;
        for (;;) {
            const int64_t p = base - lane;
            int kind;  // 0 not ready, 1 aggregate, 2 inclusive
            Span64 mine{0, 0, 0, 0};
            Carry inc{0, -1, 0};
            if (p < 0) {
                kind = 2;  // before the file: outside strings, level -1
            } else {
                const unsigned long long a = ld_acquire(states + 3 * p + 1);
                if (tagged(a, epoch)) {
                    const unsigned long long b = ld_acquire(states + 3 * p + 2);
                    if (tagged(b, epoch)) {
                        kind = 2;
                        inc.s = static_cast<int>((a >> 47) & 1);
                        inc.d = static_cast<int64_t>(a & ((1ull << 47) - 1)) - (1ll << 46);
                        inc.nl = static_cast<int64_t>(b & kPayload48);
                    } else {
                        kind = 0;
                    }
                } else {
                    const unsigned long long g = ld_acquire(states + 3 * p);
                    if (tagged(g, epoch)) {
                        kind = 1;
                        mine = widen(unpack_agg(g));
                    } else {
                        kind = 0;
                    }
                }
            }
            const unsigned inc_mask = __ballot_sync(~0u, kind == 2);
            const unsigned none_mask = __ballot_sync(~0u, kind == 0);
            const int first = inc_mask ? __ffs(inc_mask) - 1 : 32;
            const unsigned need = first == 32 ? ~0u : ((1u << first) - 1);
            if (none_mask & need) {
                ++polls;
                // Give up after the poll budget, or at once when another tile
                // already gave up (its successors would wait for it too).
                const bool expired = polls > kMaxPolls ||
                                     ((polls & 1023u) == 0 && (ld_acquire(status + 1) & kFatalErrors) != 0);
                if (expired) {
                    if (lane == 0) atomicOr(status + 1, kErrLookbackTimeout);
                    break;  // the host reports the error; outputs are not valid
                }
                __nanosleep(64);
                continue;
            }
            if (lane >= first) mine = Span64{0, 0, 0, 0};
            // lane 0 <- compose(lane 31, ..., lane 0): higher lanes are earlier tiles
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const Span64 o = shfl_span64_down(mine, off);
                if (lane + off < 32) mine = compose64(o, mine);
            }
            const Span64 window = Span64{__shfl_sync(~0u, mine.q, 0), __shfl_sync(~0u, mine.dd0, 0),
                                         __shfl_sync(~0u, mine.ddt, 0), __shfl_sync(~0u, mine.nl, 0)};
            acc = compose64(window, acc);
            if (first < 32) {
                Carry c{__shfl_sync(~0u, inc.s, first), __shfl_sync(~0u, inc.d, first),
                        __shfl_sync(~0u, inc.nl, first)};
                before = apply(c, acc);
                break;
            }
            base -= 32;
        }
    }
    if (lane == 0) {
        const Carry after = apply(before, widen(agg));
        st_release(states + 3 * t + 2, tag(epoch, static_cast<unsigned long long>(after.nl)));
        st_release(states + 3 * t + 1,
                   tag(epoch, (static_cast<unsigned long long>(after.s & 1) << 47) |
                                  static_cast<unsigned long long>(after.d + (1ll << 46))));
    }
    return before;
}

struct __align__(128) Shared {
    // a tile's bytes (TMA destination); once classified, each thread's 64
    // bytes hold its word's state until the word's stores (stash_word)
    uint8_t buf[2][kTile];
    uint64_t bar[2];
    Span warp_total[kWarps];
    int64_t next_tile;
    int esc_parity[2];  // escape state of each buffered tile's first byte
    // state before the tile in each buffer (its look-back's result)
    int carry_s[2];
    int64_t carry_d[2], carry_nl[2];
};

// What a word's stores need once the state before its tile is known, kept
// in the word's own 64 bytes of the tile buffer: eight 8-byte cells, rotated
// by the thread so that a half-warp's accesses to one cell spread over the
// banks.
struct WordState {
    uint64_t open, close, structural, newline, p0;
    Span excl;  // composed effect of the tile's words before this one
};

__device__ __forceinline__ uint64_t* state_cell(uint8_t* buf, int tid, int c) {
    return reinterpret_cast<uint64_t*>(buf + 64 * tid + 8 * ((c + tid) & 7));
}

__device__ __forceinline__ void stash_word(uint8_t* buf, int tid, const WordState& w) {
    *state_cell(buf, tid, 0) = w.open;
    *state_cell(buf, tid, 1) = w.close;
    *state_cell(buf, tid, 2) = w.structural;
    *state_cell(buf, tid, 3) = w.newline;
    *state_cell(buf, tid, 4) = w.p0;
    *state_cell(buf, tid, 5) = static_cast<uint32_t>(w.excl.dd0) | (static_cast<uint64_t>(static_cast<uint32_t>(w.excl.ddt)) << 32);
    *state_cell(buf, tid, 6) = static_cast<uint32_t>(w.excl.nl) | (static_cast<uint64_t>(static_cast<uint32_t>(w.excl.q)) << 32);
}

__device__ __forceinline__ WordState unstash_word(uint8_t* buf, int tid) {
    WordState w;
    w.open = *state_cell(buf, tid, 0);
    w.close = *state_cell(buf, tid, 1);
    w.structural = *state_cell(buf, tid, 2);
    w.newline = *state_cell(buf, tid, 3);
    w.p0 = *state_cell(buf, tid, 4);
    const uint64_t a = *state_cell(buf, tid, 5), b = *state_cell(buf, tid, 6);
    w.excl.dd0 = static_cast<int32_t>(static_cast<uint32_t>(a));
    w.excl.ddt = static_cast<int32_t>(static_cast<uint32_t>(a >> 32));
    w.excl.nl = static_cast<int32_t>(static_cast<uint32_t>(b));
    w.excl.q = static_cast<int32_t>(static_cast<uint32_t>(b >> 32));
    return w;
}

// The stores of this thread's word of tile t (state stashed in buffer bb):
// its string-index word, its words of the leveled bitmaps, its newline
// offsets.
template <int LV>
__device__ __forceinline__ void store_word(const IndexParams& p, Shared& sh, int bb, int64_t t, int tid) {
    const int64_t ws = t * kTile + 64 * tid;
    const int64_t left = p.n - ws;
    const int valid = left <= 0 ? 0 : (left >= 64 ? 64 : static_cast<int>(left));
    if (valid > 0) {
        const WordState w = unstash_word(sh.buf[bb], tid);
        const int s0 = sh.carry_s[bb];
        const int s_w = s0 ^ w.excl.q;
        const int64_t d_w = sh.carry_d[bb] + (s0 ? (w.excl.ddt - w.excl.dd0) : w.excl.dd0);
        uint64_t in_str = w.p0 ^ (s_w ? ~0ull : 0ull);
        if (valid < 64) in_str &= (1ull << valid) - 1;
        const int64_t word = ws >> 6;
        p.string_index[word] = in_str;

        uint64_t lv[LV];
        split_levels<LV>(w.open & ~in_str, w.close & ~in_str, w.structural & ~in_str, d_w, lv);
#pragma unroll
        for (int l = 0; l < LV; l++)
            if (l < p.num_levels) p.leveled[p.level_size * l + word] = lv[l];

        uint64_t nm = w.newline;
        int64_t idx = 1 + sh.carry_nl[bb] + w.excl.nl;
        while (nm) {
            const int bit = ctz64(nm);
            if (idx < p.newline_cap) p.newlines[idx] = ws + bit;
            ++idx;
            nm &= nm - 1;
        }
    }
    if (t == 0 && tid == 0 && p.newline_cap > 0) p.newlines[0] = 0;
}

// Thread 0: claim a tile and start loading it into buffer `b`.
__device__ int64_t claim_and_load(const IndexParams& p, Shared& sh, int b) {
    const int64_t t = static_cast<int64_t>(atomicAdd(p.tile_counter, 1u));
    if (t < p.ntiles) {
        const int64_t start = t * kTile;
        const int64_t bytes = p.n - start < kTile ? p.n - start : kTile;
        const uint32_t bulk = static_cast<uint32_t>(bytes & ~static_cast<int64_t>(15));
        fence_proxy_async_smem();
        if (bulk > 0) {
            mbar_arrive_expect_tx(&sh.bar[b], bulk);
            tma_load_1d(sh.buf[b], p.file + start, bulk, &sh.bar[b]);
        } else {
            mbar_arrive(&sh.bar[b]);
        }
        for (int64_t i = bulk; i < bytes; i++) sh.buf[b][i] = p.file[start + i];  // < 16 tail bytes
        sh.esc_parity[b] = start == 0 ? 0 : escape_parity_before(p.file, start);
    }
    return t;
}

// Bound by the latency of the tile's copy and its look-back, so resident
// CTAs matter more than registers: 6 per SM (shared memory's limit with two
// 16 KiB buffers) for up to eight levels, though ptxas then spills a few
// bytes; 4 with 16 levels, whose level array would spill much more.
template <int LV>
__global__ void __launch_bounds__(kThreads, LV <= 8 ? 6 : 4) index_kernel(IndexParams p) {
    __shared__ Shared sh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        mbar_init(&sh.bar[0], 1);
        mbar_init(&sh.bar[1], 1);
        fence_mbar_init();
        sh.next_tile = claim_and_load(p, sh, 0);
    }
    __syncthreads();
    int64_t t = sh.next_tile;
    int64_t t_prev = -1;  // the tile in buffer b ^ 1 whose words are still to be written
    uint32_t phase[2] = {0, 0};
    int b = 0;
    while (t < p.ntiles) {
        if (!mbar_wait_bounded(&sh.bar[b], phase[b])) {
            if (tid == 0) atomicOr(p.status + 1, kErrCopyTimeout);
        }
        phase[b] ^= 1;

        const int64_t tile_start = t * kTile;
        const int64_t ws = tile_start + 64 * tid;
        const int64_t left = p.n - ws;
        const int valid = left <= 0 ? 0 : (left >= 64 ? 64 : static_cast<int>(left));

        // ---- load and classify this thread's 64 bytes ---------------------
        // The two 32-byte halves are read in an order that depends on the
        // thread so a quarter-warp touches more shared-memory banks.
        const int rot = (tid >> 1) & 1;
        const uint4* src = reinterpret_cast<const uint4*>(sh.buf[b] + 64 * tid);
        uint32_t v[16];
        {
            const uint4 q0 = src[2 * rot], q1 = src[2 * rot + 1];
            const uint4 q2 = src[2 * (rot ^ 1)], q3 = src[2 * (rot ^ 1) + 1];
            v[0] = q0.x, v[1] = q0.y, v[2] = q0.z, v[3] = q0.w;
            v[4] = q1.x, v[5] = q1.y, v[6] = q1.z, v[7] = q1.w;
            v[8] = q2.x, v[9] = q2.y, v[10] = q2.z, v[11] = q2.w;
            v[12] = q3.x, v[13] = q3.y, v[14] = q3.z, v[15] = q3.w;
        }
        if (valid < 64) {
            // zero bytes past the end of the file (the half order is rotated)
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const int half = k >> 3;
                const int byte0 = 32 * (half ^ rot) + 4 * (k & 7);
                const int keep = valid - byte0;
                v[k] = keep >= 4 ? v[k] : (keep <= 0 ? 0u : (v[k] & ((1u << (8 * keep)) - 1)));
            }
        }
        ClassMasks m;
        {
            uint32_t b0, q0, n0, o0, c0, s0, k0, b1, q1, n1, o1, c1, s1, k1;
            classify32(v, b0, q0, n0, o0, c0, s0, k0);
            classify32(v + 8, b1, q1, n1, o1, c1, s1, k1);
            if (rot) {  // first classified half is the upper 32 bytes
                m.backslash = (static_cast<uint64_t>(b0) << 32) | b1;
                m.quote = (static_cast<uint64_t>(q0) << 32) | q1;
                m.newline = (static_cast<uint64_t>(n0) << 32) | n1;
                m.open = (static_cast<uint64_t>(o0) << 32) | o1;
                m.close = (static_cast<uint64_t>(c0) << 32) | c1;
                m.structural = (static_cast<uint64_t>(s0) << 32) | s1;
            } else {
                m.backslash = (static_cast<uint64_t>(b1) << 32) | b0;
                m.quote = (static_cast<uint64_t>(q1) << 32) | q0;
                m.newline = (static_cast<uint64_t>(n1) << 32) | n0;
                m.open = (static_cast<uint64_t>(o1) << 32) | o0;
                m.close = (static_cast<uint64_t>(c1) << 32) | c0;
                m.structural = (static_cast<uint64_t>(s1) << 32) | s0;
            }
        }

        // ---- escapes -------------------------------------------------------
        // Escape state of the first byte = parity of the backslash run ending
        // at the previous byte: from the previous word's trailing run unless
        // that word is all backslashes (or this is a warp's first lane).
        const bool all_bs = m.backslash == ~0ull;
        const int trail_par = all_bs ? 0 : (clz64(~m.backslash) & 1);
        const int prev_par = __shfl_up_sync(~0u, trail_par, 1);
        const int prev_all = __shfl_up_sync(~0u, all_bs ? 1 : 0, 1);
        int cin;
        if (lane > 0 && !prev_all) {
            cin = prev_par;
        } else {
            int run = 0, k = 64 * tid - 1;
            while (k >= 0 && sh.buf[b][k] == '\\') {
                ++run;
                --k;
            }
            cin = run & 1;
            if (k < 0) cin ^= sh.esc_parity[b];
        }
        uint32_t unused;
        const uint64_t esc = escaped_mask(m.backslash, static_cast<uint32_t>(cin), &unused);
        const uint64_t quotes = m.quote & ~esc;
        const uint64_t p0 = prefix_xor(quotes);  // in-string, word entered outside

        // ---- word summary and tile scan ------------------------------------
        Span mine;
        mine.q = popc64(quotes) & 1;
        mine.dd0 = popc64(m.open & ~p0) - popc64(m.close & ~p0);
        mine.ddt = popc64(m.open) - popc64(m.close);
        mine.nl = popc64(m.newline);
        Span incl = mine;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const Span o = shfl_span_up(incl, off);
            if (lane >= off) incl = span_compose(o, incl);
        }
        if (lane == 31) sh.warp_total[warp] = incl;
        Span excl = shfl_span_up(incl, 1);
        if (lane == 0) excl = span_identity();
        __syncthreads();
        Span warp_prefix = span_identity();
        for (int w = 0; w < warp; w++) warp_prefix = span_compose(warp_prefix, sh.warp_total[w]);
        excl = span_compose(warp_prefix, excl);

        // every byte of buffer b is read: each word's state goes into its bytes
        stash_word(sh.buf[b], tid, WordState{m.open, m.close, m.structural, m.newline, p0, excl});

        // Warp 0 looks back for this tile while the other warps write the
        // previous tile's words (its state before was found one round ago);
        // warp 0 writes its own words of it after the look-back.
        if (warp == 0) {
            Span tile_total = span_identity();
#pragma unroll
            for (int w = 0; w < kWarps; w++) tile_total = span_compose(tile_total, sh.warp_total[w]);
            const Carry before = look_back(p.tile_state, t, tile_total, p.epoch, p.status);
            if (lane == 0) {
                sh.carry_s[b] = before.s;
                sh.carry_d[b] = before.d;
                sh.carry_nl[b] = before.nl;
                if (t == p.ntiles - 1) p.status[0] = static_cast<unsigned long long>(before.nl + tile_total.nl + 1);
            }
        }
        if (t_prev >= 0) store_word<LV>(p, sh, b ^ 1, t_prev, tid);
        __syncthreads();  // buffer b ^ 1 is free; this tile's carries are set
        // Claim the next tile only now and start its copy into the other
        // buffer: a claimed tile is processed right away, so successors never
        // wait on a tile whose owner is still busy with an earlier one.
        if (tid == 0) sh.next_tile = claim_and_load(p, sh, b ^ 1);
        __syncthreads();  // the next tile's number is visible
        t_prev = t;
        t = sh.next_tile;
        b ^= 1;
    }
    // the last tile's words
    if (t_prev >= 0) store_word<LV>(p, sh, b ^ 1, t_prev, tid);
}

}  // namespace

int index_kernel_max_ctas_per_sm(int lv) {
    int blocks = 0;
    cudaError_t e;
    if (lv <= 4)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, index_kernel<4>, kThreads, 0);
    else if (lv <= 8)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, index_kernel<8>, kThreads, 0);
    else
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, index_kernel<16>, kThreads, 0);
    return e == cudaSuccess ? blocks : -1;
}

cudaError_t launch_index_kernel(const IndexParams& p, int grid, cudaStream_t stream) {
    if (p.num_levels <= 4)
        index_kernel<4><<<grid, kThreads, 0, stream>>>(p);
    else if (p.num_levels <= 8)
        index_kernel<8><<<grid, kThreads, 0, stream>>>(p);
    else
        index_kernel<16><<<grid, kThreads, 0, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace gpj
