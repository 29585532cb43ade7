// Newline index from the standalone index kernel's newline bitmap and
// per-tile newline counts: the reference's newline index ([0] = 0, then the
// offset of every '\n' in order; Sequential.java:14-34, built on the GPU by
// CombinedIndex.java:117-151 with a host-side scan of per-chunk counts).
//
// offsets: one CTA scans the tile counts (each thread sums a contiguous run
// of tiles, a block scan combines them).  scatter: a warp per tile, each
// lane taking six consecutive bitmap words, writes the tile's positions at
// the tile's offset.
#include <cstdint>

#include "index_kernel.h"
#include "word_ops.cuh"

namespace gpj {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kTileWordsL = static_cast<int>(kLineTileBytes / 64);  // 192
constexpr int kWordsPerLane = kTileWordsL / 32;                      // 6
static_assert(kWordsPerLane * 32 == kTileWordsL, "a tile's words split evenly over a warp");

__global__ void __launch_bounds__(kScanThreads) newline_offsets_kernel(const int32_t* counts, int64_t ntiles,
                                                                       int64_t* offsets,
                                                                       unsigned long long* status) {
    __shared__ int64_t warp_total[kScanThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t per = (ntiles + kScanThreads - 1) / kScanThreads;
    const int64_t b = tid * per;
    const int64_t e = b + per < ntiles ? b + per : ntiles;
    int64_t sum = 0;
    for (int64_t i = b; i < e; i++) sum += counts[i];
    int64_t incl = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int64_t o = __shfl_up_sync(~0u, incl, off);
        if (lane >= off) incl += o;
    }
    if (lane == 31) warp_total[warp] = incl;
    __syncthreads();
    int64_t before = 0, all = 0;
    for (int w = 0; w < kScanThreads / 32; w++) {
        if (w < warp) before += warp_total[w];
        all += warp_total[w];
    }
    int64_t run = before + incl - sum;
    for (int64_t i = b; i < e; i++) {
        offsets[i] = run;
        run += counts[i];
    }
    if (tid == 0) status[0] = static_cast<unsigned long long>(all + 1);
}

__global__ void __launch_bounds__(256) newline_scatter_kernel(const uint64_t* bits, int64_t words,
                                                              const int64_t* offsets, int64_t ntiles,
                                                              int64_t* newlines, int64_t cap) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    if (blockIdx.x == 0 && threadIdx.x == 0 && cap > 0) newlines[0] = 0;
    for (int64_t t = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); t < ntiles;
         t += warps) {
        const int64_t w0 = t * kTileWordsL + lane * kWordsPerLane;
        uint64_t m[kWordsPerLane];
        int cnt = 0;
#pragma unroll
        for (int i = 0; i < kWordsPerLane; i++) {
            m[i] = w0 + i < words ? bits[w0 + i] : 0ull;
            cnt += popc64(m[i]);
        }
        int incl = cnt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int o = __shfl_up_sync(~0u, incl, off);
            if (lane >= off) incl += o;
        }
        int64_t idx = 1 + offsets[t] + (incl - cnt);
#pragma unroll
        for (int i = 0; i < kWordsPerLane; i++) {
            uint64_t x = m[i];
            while (x) {
                if (idx < cap) newlines[idx] = ((w0 + i) << 6) + ctz64(x);
                ++idx;
                x &= x - 1;
            }
        }
    }
}

}  // namespace

cudaError_t launch_newline_index(const IndexParams& p, int64_t* offsets, int grid, cudaStream_t stream) {
    const int64_t ntiles = (p.n + kLineTileBytes - 1) / kLineTileBytes;
    newline_offsets_kernel<<<1, kScanThreads, 0, stream>>>(p.tile_newlines, ntiles, offsets, p.status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    newline_scatter_kernel<<<grid, 256, 0, stream>>>(p.newline_bits, p.level_size, offsets, ntiles, p.newlines,
                                                     p.newline_cap);
    return cudaGetLastError();
}

}  // namespace gpj
