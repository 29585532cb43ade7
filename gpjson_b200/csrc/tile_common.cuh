// Building blocks shared by the index kernels: one 64-byte word per thread
// of a 256-thread CTA, 16 KiB of input per round held in shared memory.
#pragma once

#include <cstdint>

#include "device_common.cuh"
#include "word_ops.cuh"

namespace gpj {

constexpr int kTileThreads = 256;
constexpr int kTileWarps = kTileThreads / 32;
constexpr int kRoundBytes = kTileThreads * 64;  // 16 KiB

// Bits of a word whose bytes lie in [lo, hi) (word-relative, may be outside 0..64).
__device__ __forceinline__ uint64_t bits_between(int64_t lo, int64_t hi) {
    if (hi <= 0 || lo >= 64 || lo >= hi) return 0;
    const uint64_t upper = hi >= 64 ? ~0ull : ((1ull << hi) - 1);
    const uint64_t lower = lo <= 0 ? 0ull : ((1ull << lo) - 1);
    return upper & ~lower;
}

// Loads word `w` (64 bytes at buf + 64w) and classifies it.  With kRotate
// (consecutive threads on consecutive words) the two 32-byte halves are read
// in a thread-dependent order so a quarter-warp of 16-byte loads spreads
// over more banks; the halves are put back in place.
template <bool kRotate = true>
__device__ __forceinline__ ClassMasks load_classify(const uint8_t* buf, int w) {
    const int rot = kRotate ? (w >> 1) & 1 : 0;
    const uint4* src = reinterpret_cast<const uint4*>(buf + 64 * w);
    uint32_t v[16];
    const uint4 q0 = src[2 * rot], q1 = src[2 * rot + 1];
    const uint4 q2 = src[2 * (rot ^ 1)], q3 = src[2 * (rot ^ 1) + 1];
    v[0] = q0.x, v[1] = q0.y, v[2] = q0.z, v[3] = q0.w;
    v[4] = q1.x, v[5] = q1.y, v[6] = q1.z, v[7] = q1.w;
    v[8] = q2.x, v[9] = q2.y, v[10] = q2.z, v[11] = q2.w;
    v[12] = q3.x, v[13] = q3.y, v[14] = q3.z, v[15] = q3.w;
    uint32_t b0, qa, n0, o0, c0, s0, k0, b1, qb, n1, o1, c1, s1, k1;
    classify32(v, b0, qa, n0, o0, c0, s0, k0);
    classify32(v + 8, b1, qb, n1, o1, c1, s1, k1);
    auto join = [rot](uint32_t first, uint32_t second) {
        return rot ? ((static_cast<uint64_t>(first) << 32) | second)
                   : ((static_cast<uint64_t>(second) << 32) | first);
    };
    ClassMasks m;
    m.backslash = join(b0, b1);
    m.quote = join(qa, qb);
    m.newline = join(n0, n1);
    m.open = join(o0, o1);
    m.close = join(c0, c1);
    m.structural = join(s0, s1);
    m.colon = join(k0, k1);
    return m;
}

__device__ __forceinline__ void restrict_masks(ClassMasks& m, uint64_t keep) {
    m.backslash &= keep;
    m.quote &= keep;
    m.newline &= keep;
    m.open &= keep;
    m.close &= keep;
    m.structural &= keep;
    m.colon &= keep;
}

// Escape state of the first byte of word w (parity of the backslash run that
// ends just before it).  Taken from the previous word's trailing run through
// a shuffle; the first lane of a warp, or a word after an all-backslash
// word, scans the bytes before it in shared memory down to `floor` (a byte
// index in buf) and adds `parity_at_floor` (the escape state of byte floor)
// when the run reaches it.  Must be called by all 32 lanes.
// Escape state of byte 64w from the bytes before it in buf: parity of the
// backslash run ending at byte 64w - 1, scanned down to `floor` (plus
// `parity_at_floor` when the run reaches it).
__device__ __forceinline__ uint32_t escape_scan_back(const uint8_t* buf, int w, int floor, int parity_at_floor) {
    int run = 0, k = 64 * w - 1;
    while (k >= floor && buf[k] == '\\') {
        ++run;
        --k;
    }
    int c = run & 1;
    if (k < floor) c ^= parity_at_floor;
    return static_cast<uint32_t>(c);
}

__device__ __forceinline__ uint32_t escape_carry_in(const uint8_t* buf, int w, uint64_t backslash, int floor,
                                                    int parity_at_floor) {
    const int lane = threadIdx.x & 31;
    const bool all_bs = backslash == ~0ull;
    const int trail_par = all_bs ? 0 : (clz64(~backslash) & 1);
    const int prev_par = __shfl_up_sync(~0u, trail_par, 1);
    const int prev_all = __shfl_up_sync(~0u, all_bs ? 1 : 0, 1);
    if (lane > 0 && !prev_all) return static_cast<uint32_t>(prev_par);
    return escape_scan_back(buf, w, floor, parity_at_floor);
}

__device__ __forceinline__ Span shfl_span_up(const Span& v, int off) {
    return Span{__shfl_up_sync(~0u, v.q, off), __shfl_up_sync(~0u, v.dd0, off), __shfl_up_sync(~0u, v.ddt, off),
                __shfl_up_sync(~0u, v.nl, off)};
}

// Exclusive compose-scan of one Span per thread across the CTA, in thread
// order.  `scratch` holds kTileWarps Spans.  Contains one __syncthreads; the
// caller must barrier before `scratch` is reused.
__device__ __forceinline__ Span block_scan_span(Span mine, Span* scratch, Span* total) {
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
    __syncthreads();
    Span prefix = span_identity();
    Span all = span_identity();
#pragma unroll
    for (int w = 0; w < kTileWarps; w++) {
        if (w == warp) prefix = all;
        all = span_compose(all, scratch[w]);
    }
    *total = all;
    return span_compose(prefix, excl);
}

// Exclusive sum of an int and minimum of an int64 across the CTA.  One
// __syncthreads; `isum` holds kTileWarps ints, `imin` kTileWarps int64.
__device__ __forceinline__ int block_sum_min(int x, int64_t y, int* isum, int64_t* imin, int* total,
                                             int64_t* minimum) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = x;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int o = __shfl_up_sync(~0u, incl, off);
        if (lane >= off) incl += o;
    }
    int64_t mn = y;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const int64_t o = __shfl_xor_sync(~0u, mn, off);
        mn = o < mn ? o : mn;
    }
    if (lane == 31) isum[warp] = incl;
    if (lane == 0) imin[warp] = mn;
    __syncthreads();
    int before = 0, all = 0;
    int64_t m = imin[0];
#pragma unroll
    for (int w = 0; w < kTileWarps; w++) {
        if (w < warp) before += isum[w];
        all += isum[w];
        m = imin[w] < m ? imin[w] : m;
    }
    *total = all;
    *minimum = m;
    return before + incl - x;
}

}  // namespace gpj
