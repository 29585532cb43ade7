// Newline index from the standalone index kernel's newline bitmap and
// per-tile newline counts: the reference's newline index ([0] = 0, then the
// offset of every '\n' in order; Sequential.java:14-34, built on the GPU by
// CombinedIndex.java:117-151 with a host-side scan of per-chunk counts).
//
// offsets: block scans of the tile counts, 1024 tiles per CTA.  scatter: a
// warp per tile adds the sums of the earlier blocks to the tile's offset and
// writes its positions, each lane taking consecutive bitmap words.
#include <cstdint>

#include "index_kernel.h"
#include "word_ops.cuh"

namespace gpj {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kTileWordsL = static_cast<int>(kLineTileBytes / 64);  // 224
constexpr int kWordsPerLane = kTileWordsL / 32;                      // 7
static_assert(kWordsPerLane * 32 == kTileWordsL, "a tile's words split evenly over a warp");

// Offsets of the tile counts within blocks of 1024 tiles (coalesced, one
// CTA per block); the block sums go after the ntiles entries.
__global__ void __launch_bounds__(kScanThreads) newline_offsets_kernel(const int32_t* counts, int64_t ntiles,
                                                                       int64_t* offsets) {
    __shared__ int64_t warp_total[kScanThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kScanThreads + tid;
    const int64_t c = i < ntiles ? counts[i] : 0;
    int64_t incl = c;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int64_t o = __shfl_up_sync(~0u, incl, off);
        if (lane >= off) incl += o;
    }
    if (lane == 31) warp_total[warp] = incl;
    __syncthreads();
    int64_t before = 0, all = 0;
#pragma unroll 8
    for (int w = 0; w < kScanThreads / 32; w++) {
        if (w < warp) before += warp_total[w];
        all += warp_total[w];
    }
    if (i < ntiles) offsets[i] = before + incl - c;
    if (tid == 0) offsets[ntiles + blockIdx.x] = all;
}

// A warp per tile: the sum of the earlier blocks (lanes add them up), the
// tile's offset in its block, then the positions, each lane taking
// consecutive bitmap words.
__global__ void __launch_bounds__(256) newline_scatter_kernel(const uint64_t* bits, int64_t words,
                                                              const int32_t* counts, const int64_t* offsets,
                                                              int64_t ntiles, int64_t* newlines, int64_t cap,
                                                              unsigned long long* status) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    const int64_t* block_sums = offsets + ntiles;
    if (blockIdx.x == 0 && threadIdx.x == 0 && cap > 0) newlines[0] = 0;
    for (int64_t t = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); t < ntiles;
         t += warps) {
        const int64_t blk = t / kScanThreads;
        int64_t base = 0;
        for (int64_t b = lane; b < blk; b += 32) base += block_sums[b];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) base += __shfl_xor_sync(~0u, base, off);
        base += offsets[t];
        if (t == ntiles - 1 && lane == 0) status[0] = static_cast<unsigned long long>(base + counts[t] + 1);
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
        int64_t idx = 1 + base + (incl - cnt);
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
    const int64_t blocks = (ntiles + kScanThreads - 1) / kScanThreads;
    newline_offsets_kernel<<<static_cast<unsigned>(blocks), kScanThreads, 0, stream>>>(p.tile_newlines, ntiles, offsets);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    newline_scatter_kernel<<<grid, 256, 0, stream>>>(p.newline_bits, p.level_size, p.tile_newlines, offsets, ntiles,
                                                     p.newlines, p.newline_cap, p.status);
    return cudaGetLastError();
}

}  // namespace gpj
