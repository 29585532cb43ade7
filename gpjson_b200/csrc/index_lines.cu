// Line-parallel structural index for NDJSON on sm_100a, with the JSONPath
// queries evaluated in the same pass (the fast path).
//
// In newline-delimited JSON every line is a complete value, so at each
// '\n' the reference's scan state (Sequential.java:36-128: inside-string
// flag, level counter, escape flag) is (outside, -1, clear) again.  This
// kernel uses that: the CTA that claims a 16 KiB tile builds the index of
// every line that starts in it, starting each line from that state, and runs
// on past the tile end to finish its last line.  No string or level carry
// crosses tiles, so CTAs depend on each other only through the newline
// count, which a wide decoupled look-back resolves after the tile's work.
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
// Fused queries: the final string and level masks of the tile and of the
// first 16 KiB past it stay in shared memory next to the bytes, so the CTA
// runs the find_value interpreter (interp.cuh) on its own lines there, one
// (line, query) pair per thread, and writes the offsets.  Lines that do not
// fit (or whose evaluation would read past the bytes held) are flagged as
// deferred and the host evaluates them with the find_value kernel.
#include <cstdint>

#include "device_common.cuh"
#include "index_kernel.h"
#include "interp.cuh"
#include "tile_common.cuh"
#include "word_ops.cuh"

namespace gpj {

namespace {

constexpr int64_t kTile = kRoundBytes;  // 16 KiB
constexpr int kTileWords = kTile / 64;  // 256
constexpr int kSmemWords = 2 * kTileWords;  // tile + first extension chunk
constexpr int64_t kNone = INT64_MAX;
// Longest run past the tile end a CTA follows to finish its last line; a
// longer line sends the whole input to the exact kernel.
constexpr int64_t kMaxExtension = 8ll << 20;
// Lines of one tile whose starts are kept for the fused queries.
constexpr int kMaxTileLines = 1024;
constexpr unsigned long long kPayload48 = (1ull << 48) - 1;

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
                polls > kMaxPolls || ((polls & 1023u) == 0 && ld_acquire(status + 1) != 0);
            if (expired) {
                if (lane == 0) atomicOr(status + 1, kErrLookbackTimeout);
                break;
            }
            __nanosleep(32);
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

// Shared memory of one CTA (dynamic; LV level rows of masks).
template <int LV>
struct LShared {
    uint8_t buf[2][kTile];              // tile, then the first extension chunk (contiguous)
    uint64_t str[kSmemWords];           // final in-string masks of those words
    uint64_t colon[kSmemWords];         // ':' outside strings
    uint64_t lv[LV][kSmemWords];        // final level masks
    int32_t nlpos[kMaxTileLines];       // offsets of the tile's first newlines
    uint64_t bar[2];
    Span span_scratch[kTileWarps];
    int isum[kTileWarps];
    int64_t imin[kTileWarps];
    int64_t tile;
    int64_t ext_end;  // b_t
    int64_t nl_before;
    int64_t smem_hi;  // bytes [tile_start, smem_hi) have final masks in shared memory
    int carry_s, carry_esc;
    int64_t carry_d;
};

// Issues the TMA load of [start, start + bytes) into `dst` on `bar` (thread 0).
__device__ __forceinline__ void load_round(const uint8_t* file, int64_t start, int64_t bytes, uint8_t* dst,
                                           uint64_t* bar) {
    const uint32_t bulk = static_cast<uint32_t>(bytes & ~static_cast<int64_t>(15));
    fence_proxy_async_smem();
    if (bulk > 0) {
        mbar_arrive_expect_tx(bar, bulk);
        tma_load_1d(dst, file + start, bulk, bar);
    } else {
        mbar_arrive(bar);
    }
    for (int64_t i = bulk; i < bytes; i++) dst[i] = file[start + i];
}

// Final masks of one word: checks the '\n' bits in `check`, stores the word
// to shared memory at `slot` (>= 0) and to the global index when `owned`.
template <int LV>
__device__ __forceinline__ void finish_word(const IndexParams& p, LShared<LV>& sh, const ClassMasks& m, uint64_t p0,
                                            int s_w, int64_t d_w, int64_t word, bool owned, int slot,
                                            uint64_t valid, uint64_t check) {
    const uint64_t in_str = (p0 ^ (s_w ? ~0ull : 0ull)) & valid;
    const uint64_t open = m.open & ~in_str, close = m.close & ~in_str;
    if (check) {
        // every checked '\n' must be outside strings at level -1
        if (check & in_str) atomicOr(p.status + 1, kErrIrregular);
        uint64_t c = check;
        while (c) {
            const int bit = ctz64(c);
            const uint64_t below = (1ull << bit) - 1;
            const int64_t d = d_w + popc64(open & below) - popc64(close & below);
            if (d != -1) atomicOr(p.status + 1, kErrIrregular);
            c &= c - 1;
        }
    }
    if (!owned && slot < 0) return;
    uint64_t lv[LV];
    split_levels<LV>(open, close, m.structural & ~in_str, d_w, lv);
    if (slot >= 0) {
        sh.str[slot] = in_str;
        sh.colon[slot] = m.colon & ~in_str;
#pragma unroll
        for (int l = 0; l < LV; l++) sh.lv[l][slot] = lv[l];
    }
    if (owned && p.materialize) {
        p.string_index[word] = in_str;
#pragma unroll
        for (int l = 0; l < LV; l++)
            if (l < p.num_levels) p.leveled[p.level_size * l + word] = lv[l];
    }
}

template <int LV>
__global__ void __launch_bounds__(kTileThreads) line_index_kernel(IndexParams p) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    LShared<LV>& sh = *reinterpret_cast<LShared<LV>*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    unsigned long long* nl_agg = p.tile_state;
    unsigned long long* nl_inc = p.tile_state + p.ntiles;
    if (tid == 0) {
        mbar_init(&sh.bar[0], 1);
        mbar_init(&sh.bar[1], 1);
        fence_mbar_init();
    }
    uint32_t phase0 = 0, phase1 = 0;

    for (;;) {
        __syncthreads();  // buffers and shared slots are free
        if (tid == 0) {
            const int64_t t = static_cast<int64_t>(atomicAdd(p.tile_counter, 1u));
            sh.tile = t;
            if (t < p.ntiles) {
                const int64_t start = t * kTile;
                load_round(p.file, start, p.n - start < kTile ? p.n - start : kTile, sh.buf[0], &sh.bar[0]);
            }
        }
        __syncthreads();
        const int64_t t = sh.tile;
        if (t >= p.ntiles) break;
        if (!mbar_wait_bounded(&sh.bar[0], phase0) && tid == 0) atomicOr(p.status + 1, kErrCopyTimeout);
        phase0 ^= 1;

        const int64_t tile_start = t * kTile;
        const int64_t tile_end = p.n - tile_start < kTile ? p.n : tile_start + kTile;
        const int64_t ws = tile_start + 64 * tid;
        const uint64_t valid = bits_between(0, p.n - ws);

        // ---- round 0: the tile ---------------------------------------------
        ClassMasks m = load_classify(sh.buf[0], tid);
        restrict_masks(m, valid);
        const uint64_t my_newlines = m.newline;
        const int64_t first_local = my_newlines ? 64 * tid + ctz64(my_newlines) : kNone;
        int tile_nl = 0;
        int64_t first_nl = kNone;
        const int my_nl_excl = block_sum_min(popc64(my_newlines), first_local, sh.isum, sh.imin, &tile_nl, &first_nl);
        if (tid == 0) st_release(nl_agg + t, tag48(p.epoch, static_cast<unsigned long long>(tile_nl)));
        if (p.num_queries > 0) {
            uint64_t nm = my_newlines;
            int k = my_nl_excl;
            while (nm && k < kMaxTileLines) {
                sh.nlpos[k++] = 64 * tid + ctz64(nm);
                nm &= nm - 1;
            }
        }

        const int64_t a_t = t == 0 ? 0 : (first_nl == kNone ? kNone : tile_start + first_nl);
        if (a_t != kNone) {
            const uint64_t mine = valid & bits_between(a_t - ws, 64);
            restrict_masks(m, mine);
            const int floor = static_cast<int>(a_t - tile_start);
            const uint32_t cin = escape_carry_in(sh.buf[0], tid, m.backslash, floor, 0);
            uint32_t cout;
            const uint64_t esc = escaped_mask(m.backslash, cin, &cout);
            const uint64_t quotes = m.quote & ~esc;
            const uint64_t p0 = prefix_xor(quotes);
            Span sp{popc64(quotes) & 1, popc64(m.open & ~p0) - popc64(m.close & ~p0),
                    popc64(m.open) - popc64(m.close), 0};
            Span total;
            const Span ex = block_scan_span(sp, sh.span_scratch, &total);
            // lines start outside strings at level -1
            const int s_w = ex.q;
            const int64_t d_w = -1 + static_cast<int64_t>(ex.dd0);
            const uint64_t check = m.newline & ~(a_t >= ws && a_t < ws + 64 ? (1ull << (a_t - ws)) : 0ull);
            if (ws < p.n)
                finish_word<LV>(p, sh, m, p0, s_w, d_w, ws >> 6, ws >= a_t, tid, valid, check);
            if (tid == kTileThreads - 1) {
                sh.carry_s = total.q;
                sh.carry_d = -1 + static_cast<int64_t>(total.dd0);
                sh.carry_esc = static_cast<int>(cout);
            }
            if (tid == 0) {
                sh.ext_end = tile_end;
                sh.smem_hi = tile_end;
            }
            __syncthreads();

            // ---- extension: finish the last line past the tile end ------------
            if (tile_end < p.n) {
                if (warp == 0) {
                    // first '\n' at or after tile_end (16 bytes per lane per step)
                    const int lane = tid & 31;
                    int64_t found = kNone;
                    const int64_t limit = p.n - tile_end > kMaxExtension ? tile_end + kMaxExtension : p.n;
                    for (int64_t base = tile_end; base < limit && found == kNone; base += 512) {
                        const int64_t q = base + 16 * lane;
                        uint64_t nlbits = 0;
                        if (q + 16 <= p.n) {
                            const uint4 v = __ldg(reinterpret_cast<const uint4*>(p.file + q));
                            const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                            for (int i = 0; i < 4; i++) {
                                uint32_t f = eq_bytes(w4[i], 0x0A0A0A0Au);
                                while (f) {
                                    nlbits |= 1ull << (4 * i + ((__ffs(f) - 1) >> 3));
                                    f &= f - 1;
                                }
                            }
                        } else {
                            for (int64_t k = q; k < p.n; k++)
                                if (p.file[k] == '\n') nlbits |= 1ull << (k - q);
                        }
                        const int64_t mine_first = nlbits ? q + ctz64(nlbits) : kNone;
                        int64_t best = mine_first;
#pragma unroll
                        for (int off = 16; off > 0; off >>= 1) {
                            const int64_t o = __shfl_xor_sync(~0u, best, off);
                            best = o < best ? o : best;
                        }
                        found = best;
                    }
                    if (lane == 0) {
                        if (found == kNone && limit < p.n) {
                            // a very long line: leave the input to the exact kernel
                            atomicOr(p.status + 1, kErrLongLine);
                            found = tile_end;
                        }
                        sh.ext_end = found == kNone ? p.n : found;
                    }
                }
                __syncthreads();
                const int64_t b_t = sh.ext_end;
                const int64_t own_end = (b_t + 63) & ~static_cast<int64_t>(63);  // words starting before b_t
                if (b_t == tile_end) {
                    // the tile ends exactly at the next line: check the state there
                    if (tid == 0 && (sh.carry_s != 0 || sh.carry_d != -1)) atomicOr(p.status + 1, kErrIrregular);
                }
                for (int64_t cs = tile_end; cs < own_end && cs < p.n; cs += kTile) {
                    const bool first_chunk = cs == tile_end;
                    const int64_t chunk_end = own_end < p.n ? own_end : p.n;
                    const int64_t bytes = chunk_end - cs < kTile ? chunk_end - cs : kTile;
                    const int nwords = static_cast<int>((bytes + 63) >> 6);
                    if (tid == 0) load_round(p.file, cs, bytes, sh.buf[1], &sh.bar[1]);
                    if (!mbar_wait_bounded(&sh.bar[1], phase1) && tid == 0)
                        atomicOr(p.status + 1, kErrCopyTimeout);
                    phase1 ^= 1;
                    const int s_in = sh.carry_s;
                    const int64_t d_in = sh.carry_d;
                    const int esc_in = sh.carry_esc;
                    const int64_t cw = cs + 64 * tid;
                    const uint64_t cvalid = tid < nwords ? bits_between(0, cs + bytes - cw) : 0ull;
                    ClassMasks e{0, 0, 0, 0, 0, 0, 0};
                    if (tid < nwords) {
                        e = load_classify(sh.buf[1], tid);
                        restrict_masks(e, cvalid);
                    }
                    const uint32_t ecin = escape_carry_in(sh.buf[1], tid, e.backslash, 0, esc_in);
                    uint32_t ecout;
                    const uint64_t eesc = escaped_mask(e.backslash, ecin, &ecout);
                    const uint64_t equotes = e.quote & ~eesc;
                    const uint64_t ep0 = prefix_xor(equotes);
                    Span esp{popc64(equotes) & 1, popc64(e.open & ~ep0) - popc64(e.close & ~ep0),
                             popc64(e.open) - popc64(e.close), 0};
                    Span etotal;
                    const Span eex = block_scan_span(esp, sh.span_scratch, &etotal);
                    const int es_w = s_in ^ eex.q;
                    const int64_t ed_w = d_in + (s_in ? (eex.ddt - eex.dd0) : eex.dd0);
                    const uint64_t echeck = (b_t >= cw && b_t < cw + 64) ? (e.newline & (1ull << (b_t - cw))) : 0ull;
                    if (tid < nwords)
                        finish_word<LV>(p, sh, e, ep0, es_w, ed_w, cw >> 6, true,
                                        first_chunk ? kTileWords + tid : -1, cvalid, echeck);
                    __syncthreads();  // everyone read the carry and the buffer
                    if (tid == nwords - 1) {
                        sh.carry_s = s_in ^ etotal.q;
                        sh.carry_d = d_in + (s_in ? (etotal.ddt - etotal.dd0) : etotal.dd0);
                        sh.carry_esc = static_cast<int>(ecout);
                    }
                    // the bytes stay readable for the fused queries only when the
                    // whole extension fit in this one chunk
                    if (tid == 0 && first_chunk && own_end <= tile_end + kTile) sh.smem_hi = cs + bytes;
                    __syncthreads();
                }
            }
        }

        // ---- newline index ---------------------------------------------------
        if (warp == 0) {
            const int64_t before = lookback_newlines(nl_agg, nl_inc, t, tile_nl, p.epoch, p.status);
            if (tid == 0) {
                sh.nl_before = before;
                if (t == p.ntiles - 1) p.status[0] = static_cast<unsigned long long>(before + tile_nl + 1);
                if (t == 0 && p.newline_cap > 0 && p.materialize) p.newlines[0] = 0;
            }
        }
        __syncthreads();
        const int64_t nl_before = sh.nl_before;
        if (p.materialize) {
            uint64_t nm = my_newlines;
            int64_t idx = 1 + nl_before + my_nl_excl;
            while (nm) {
                const int bit = ctz64(nm);
                if (idx < p.newline_cap) p.newlines[idx] = ws + bit;
                ++idx;
                nm &= nm - 1;
            }
        }

        // ---- fused queries over this tile's lines -------------------------------
        if (p.num_queries > 0 && a_t != kNone) {
            const int lines = tile_nl + (t == 0 ? 1 : 0);
            if (tile_nl > kMaxTileLines) {
                if (tid == 0) atomicOr(p.status + 1, kErrDeferred);
            } else {
                const int64_t b_t = sh.ext_end;
                const int64_t hi = sh.smem_hi;
                LineView view{sh.buf[0] - tile_start, p.n, sh.str - (tile_start >> 6),
                              &sh.lv[0][0] - (tile_start >> 6), kSmemWords, hi, sh.colon - (tile_start >> 6)};
                const int items = lines * p.num_queries;
                const int64_t per_line = 2 * static_cast<int64_t>(p.slots);
                for (int it = tid; it < items; it += kTileThreads) {
                    const int li = it / p.num_queries, q = it - li * p.num_queries;
                    int64_t start, end, line;
                    if (t == 0) {
                        start = li == 0 ? 0 : tile_start + sh.nlpos[li - 1];
                        line = li;
                    } else {
                        start = tile_start + sh.nlpos[li];
                        line = 1 + nl_before + li;
                    }
                    const int nxt = t == 0 ? li : li + 1;  // index in nlpos of the next line's start
                    end = nxt < tile_nl ? tile_start + sh.nlpos[nxt] : b_t;
                    if (line >= p.out_lines) {
                        atomicOr(p.status + 1, kErrOutOverflow);
                        continue;
                    }
                    int64_t* res = p.out + (static_cast<int64_t>(q) * p.out_lines + line) * per_line;
                    for (int64_t k = 0; k < per_line; k++) res[k] = -1;
                    if (end > hi ||
                        run_line(view, start, end, p.bytecode + p.offsets[q], res) == kLineDeferred)
                        atomicOr(p.status + 1, kErrDeferred);
                }
            }
        }
    }
}

template <int LV>
cudaError_t prepare() {
    static bool done = false;
    if (done) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(line_index_kernel<LV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(sizeof(LShared<LV>)));
    if (e == cudaSuccess) done = true;
    return e;
}

template <int LV>
int occupancy() {
    if (prepare<LV>() != cudaSuccess) return -1;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, line_index_kernel<LV>, kTileThreads,
                                                      sizeof(LShared<LV>)) != cudaSuccess)
        return -1;
    return blocks;
}

template <int LV>
cudaError_t launch(const IndexParams& p, int grid, cudaStream_t stream) {
    cudaError_t e = prepare<LV>();
    if (e != cudaSuccess) return e;
    line_index_kernel<LV><<<grid, kTileThreads, sizeof(LShared<LV>), stream>>>(p);
    return cudaGetLastError();
}

}  // namespace

int line_index_max_ctas_per_sm(int lv) {
    if (lv <= 4) return occupancy<4>();
    if (lv <= 8) return occupancy<8>();
    return occupancy<16>();
}

cudaError_t launch_line_index_kernel(const IndexParams& p, int grid, cudaStream_t stream) {
    if (p.num_levels <= 4) return launch<4>(p, grid, stream);
    if (p.num_levels <= 8) return launch<8>(p, grid, stream);
    return launch<16>(p, grid, stream);
}

}  // namespace gpj
