// Newline index from the standalone index kernel's newline bitmap and
// per-tile newline counts: the reference's newline index ([0] = 0, then the
// offset of every '\n' in order; Sequential.java:14-34, built on the GPU by
// CombinedIndex.java:117-151 with a host-side scan of per-chunk counts).
//
// offsets: block scans of the tile counts, 1024 tiles per CTA.  scatter: a
// warp per tile adds the sums of the earlier blocks to the tile's offset and
// writes its positions, each lane taking consecutive bitmap words.  A batch
// of files shares one tile numbering; each file's newlines count from its
// first tile.
#include <cstdint>

#include "index_kernel.h"
#include "word_ops.cuh"

namespace gpj {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kTileWordsL = static_cast<int>(kStandaloneTileBytes / 64);  // 480
constexpr int kWordsPerLane = kTileWordsL / 32;                            // 15
static_assert(kWordsPerLane * 32 == kTileWordsL, "a tile's words split evenly over a warp");

// Offsets of the tile counts within blocks of 1024 tiles (coalesced, one
// CTA per block, blocks blk0, blk0 + 1, ...); the block sums go after the
// ntiles entries.
__global__ void __launch_bounds__(kScanThreads) newline_offsets_kernel(const int32_t* counts, int64_t ntiles,
                                                                       int64_t* offsets, int64_t blk0) {
    __shared__ int64_t warp_total[kScanThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t blk = blk0 + blockIdx.x;
    const int64_t i = blk * kScanThreads + tid;
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
    if (tid == 0) offsets[ntiles + blk] = all;
}

// Sum of the tile counts before tile t of the whole batch (all lanes of a
// warp call it; the block sums are added up by the lanes).
__device__ __forceinline__ int64_t tiles_before(const int64_t* offsets, int64_t ntiles, int64_t t) {
    const int lane = threadIdx.x & 31;
    const int64_t* block_sums = offsets + ntiles;
    const int64_t blk = t / kScanThreads;
    int64_t base = 0;
    for (int64_t b = lane; b < blk; b += 32) base += block_sums[b];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) base += __shfl_xor_sync(~0u, base, off);
    return base + offsets[t];
}

// A warp per tile of [t0, t1): the tile's newlines before it in its file
// (the batch prefix at the tile minus the prefix at the file's first tile),
// then the positions, each lane taking consecutive bitmap words.  `files`
// null: the single file `one`.  `lines_done` (optional, single file): the
// warp of tile t1 - 1 writes there how many lines have both ends in the
// newline index written so far (the newlines up to t1 - 1, plus the last
// line when t1 - 1 is the file's last tile).
__global__ void __launch_bounds__(256) newline_scatter_kernel(const int32_t* counts, const int64_t* offsets,
                                                              int64_t ntiles, int64_t t0, int64_t t1, LineFile one,
                                                              const LineFile* files, int nfiles,
                                                              int64_t* lines_done) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t t = t0 + static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); t < t1;
         t += warps) {
        LineFile F = one;
        if (files) {
            int lo = 0, hi = nfiles - 1;  // last file with tile_begin <= t
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (files[mid].tile_begin <= t)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            F = files[lo];
        }
        const int64_t lt = t - F.tile_begin;
        const int64_t base = tiles_before(offsets, ntiles, t) - tiles_before(offsets, ntiles, F.tile_begin);
        if (lt == 0 && lane == 0 && F.cap > 0) F.newlines[0] = 0;
        if (lt == F.ntiles - 1 && lane == 0) F.status[0] = static_cast<unsigned long long>(base + counts[t] + 1);
        if (lines_done && t == t1 - 1 && lane == 0) *lines_done = base + counts[t] + (lt == F.ntiles - 1 ? 1 : 0);
        const int64_t w0 = lt * kTileWordsL + lane * kWordsPerLane;
        uint64_t m[kWordsPerLane];
        int cnt = 0;
#pragma unroll
        for (int i = 0; i < kWordsPerLane; i++) {
            m[i] = w0 + i < F.words ? F.newline_bits[w0 + i] : 0ull;
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
                if (idx < F.cap) F.newlines[idx] = ((w0 + i) << 6) + ctz64(x);
                ++idx;
                x &= x - 1;
            }
        }
    }
}

}  // namespace

cudaError_t launch_newline_index_batch(const int32_t* tile_newlines, int64_t total_tiles, const LineFile* files,
                                       int nfiles, int64_t* offsets, int grid, cudaStream_t stream) {
    const int64_t blocks = (total_tiles + kScanThreads - 1) / kScanThreads;
    newline_offsets_kernel<<<static_cast<unsigned>(blocks), kScanThreads, 0, stream>>>(tile_newlines, total_tiles,
                                                                                       offsets, 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    newline_scatter_kernel<<<grid, 256, 0, stream>>>(tile_newlines, offsets, total_tiles, 0, total_tiles, LineFile{},
                                                     files, nfiles, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_newline_index_range(const IndexParams& p, int64_t* offsets, int64_t t0, int64_t t1,
                                       int64_t* lines_done, int grid, cudaStream_t stream) {
    const int64_t ntiles = (p.n + kStandaloneTileBytes - 1) / kStandaloneTileBytes;
    if (t0 % kScanThreads != 0 || t1 <= t0 || t1 > ntiles || (t1 != ntiles && t1 % kScanThreads != 0))
        return cudaErrorInvalidValue;
    const int64_t blk0 = t0 / kScanThreads;
    const int64_t blocks = (t1 - t0 + kScanThreads - 1) / kScanThreads;
    newline_offsets_kernel<<<static_cast<unsigned>(blocks), kScanThreads, 0, stream>>>(p.tile_newlines, ntiles, offsets,
                                                                                       blk0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const LineFile one{p.newline_bits, p.level_size, p.newlines, p.newline_cap, p.status, 0, ntiles};
    newline_scatter_kernel<<<grid, 256, 0, stream>>>(p.tile_newlines, offsets, ntiles, t0, t1, one, nullptr, 0,
                                                     lines_done);
    return cudaGetLastError();
}

cudaError_t launch_newline_index(const IndexParams& p, int64_t* offsets, int grid, cudaStream_t stream) {
    const int64_t ntiles = (p.n + kStandaloneTileBytes - 1) / kStandaloneTileBytes;
    return launch_newline_index_range(p, offsets, 0, ntiles, nullptr, grid, stream);
}

}  // namespace gpj
