// Device-side value extraction: the bytes of every matched value gathered
// into one compact buffer, with ResultItem's semantics
// (result/ResultItem.java:32-52): a (start, end) pair with start == -1 is
// null; otherwise the value is file[start, end).  The reference slices the
// memory-mapped file on the host, one String per access; here one pass
// over the result pairs sizes the values, a scan places them, and a copy
// kernel moves the bytes, so the host receives values without reading the
// file again.
//
// Pairs are numbered i = q * per_query + r and read at
// pairs[2 * (q * stride + r)], so query blocks of a result buffer whose line
// capacity exceeds the line count can be read in place.
#include <cstdint>

#include "values.h"

namespace gpj {

namespace {

constexpr int kValThreads = 1024;
constexpr int64_t kShortValue = 32;  // longer values are copied by a whole warp

__device__ __forceinline__ const int64_t* pair_at(const int64_t* pairs, int64_t i, int64_t per_query, int64_t stride) {
    const int64_t q = i / per_query;
    return pairs + 2 * (q * stride + (i - q * per_query));
}

// Exclusive sum of `v` over the CTA (1024 threads); *all receives the total.
__device__ __forceinline__ int64_t block_exclusive_sum(int64_t v, int64_t* warp_total, int64_t* all) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int64_t incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int64_t o = __shfl_up_sync(~0u, incl, off);
        if (lane >= off) incl += o;
    }
    if (lane == 31) warp_total[warp] = incl;
    __syncthreads();
    int64_t before = 0, sum = 0;
#pragma unroll 8
    for (int w = 0; w < kValThreads / 32; w++) {
        if (w < warp) before += warp_total[w];
        sum += warp_total[w];
    }
    *all = sum;
    return before + incl - v;
}

// Kind and length of each pair; block-local offsets and the block totals.
__global__ void __launch_bounds__(kValThreads) value_lengths_kernel(const int64_t* pairs, int64_t npairs,
                                                                    int64_t per_query, int64_t stride, int64_t n,
                                                                    uint8_t* kinds, int64_t* offsets,
                                                                    int64_t* block_sums) {
    __shared__ int64_t warp_total[kValThreads / 32];
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kValThreads + threadIdx.x;
    int64_t len = 0;
    if (i < npairs) {
        const int64_t* pr = pair_at(pairs, i, per_query, stride);
        const int64_t s = pr[0], e = pr[1];
        uint8_t kind = kValueNull;
        if (s != -1) {
            // end before start: the reference fails building byte[end - start]
            // (NegativeArraySizeException); such items are marked, not read
            if (s < 0 || e < s || e > n) {
                kind = kValueUnreadable;
            } else {
                kind = kValuePresent;
                len = e - s;
            }
        }
        kinds[i] = kind;
    }
    int64_t all;
    const int64_t excl = block_exclusive_sum(len, warp_total, &all);
    if (i < npairs) offsets[i] = excl;
    if (threadIdx.x == 0) block_sums[blockIdx.x] = all;
}

// Exclusive scan of the block totals in place (one CTA); *total = the sum.
__global__ void __launch_bounds__(kValThreads) value_block_scan_kernel(int64_t* block_sums, int64_t nblocks,
                                                                       int64_t* total) {
    __shared__ int64_t warp_total[kValThreads / 32];
    int64_t carry = 0;
    for (int64_t base = 0; base < nblocks; base += kValThreads) {
        const int64_t i = base + threadIdx.x;
        const int64_t v = i < nblocks ? block_sums[i] : 0;
        int64_t all;
        const int64_t excl = block_exclusive_sum(v, warp_total, &all);
        if (i < nblocks) block_sums[i] = carry + excl;
        carry += all;
        __syncthreads();  // warp_total is reused by the next chunk
    }
    if (threadIdx.x == 0) *total = carry;
}

// Final offsets and the bytes: a lane copies a short value itself, the warp
// copies long ones together (consecutive lanes on consecutive bytes).
// Values that would end past `cap` are not written.
__global__ void __launch_bounds__(256) value_copy_kernel(const uint8_t* file, const int64_t* pairs, int64_t npairs,
                                                         int64_t per_query, int64_t stride, const uint8_t* kinds,
                                                         int64_t* offsets, const int64_t* block_sums,
                                                         const int64_t* total, uint8_t* out, int64_t cap) {
    const int lane = threadIdx.x & 31;
    const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
    // the grid is a multiple of 32 threads, so every warp runs the loop in step
    for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < npairs;
         base += step) {
        const int64_t i = base + lane;
        int64_t off = 0, src = 0, len = 0;
        if (i < npairs) {
            off = offsets[i] + block_sums[i / kValThreads];
            offsets[i] = off;
            if (kinds[i] == kValuePresent) {
                const int64_t* pr = pair_at(pairs, i, per_query, stride);
                src = pr[0];
                len = pr[1] - pr[0];
                if (off + len > cap) len = 0;
            }
        }
        if (len <= kShortValue) {
            for (int64_t k = 0; k < len; k++) out[off + k] = file[src + k];
        }
        unsigned long_ones = __ballot_sync(~0u, len > kShortValue);
        while (long_ones) {
            const int l = __ffs(long_ones) - 1;
            long_ones &= long_ones - 1;
            const int64_t o = __shfl_sync(~0u, off, l), s = __shfl_sync(~0u, src, l), n = __shfl_sync(~0u, len, l);
            for (int64_t k = lane; k < n; k += 32) out[o + k] = file[s + k];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) offsets[npairs] = *total;
}

}  // namespace

int64_t value_scan_blocks(int64_t npairs) { return (npairs + kValThreads - 1) / kValThreads; }

cudaError_t launch_value_sizes(const int64_t* pairs, int64_t npairs, int64_t per_query, int64_t stride, int64_t n,
                               uint8_t* kinds, int64_t* offsets, int64_t* block_sums, int64_t* total,
                               cudaStream_t stream) {
    const int64_t blocks = value_scan_blocks(npairs);
    if (blocks > 0) {
        value_lengths_kernel<<<static_cast<unsigned>(blocks), kValThreads, 0, stream>>>(
            pairs, npairs, per_query, stride, n, kinds, offsets, block_sums);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    value_block_scan_kernel<<<1, kValThreads, 0, stream>>>(block_sums, blocks, total);
    return cudaGetLastError();
}

cudaError_t launch_value_copy(const uint8_t* file, const int64_t* pairs, int64_t npairs, int64_t per_query,
                              int64_t stride, const uint8_t* kinds, int64_t* offsets, const int64_t* block_sums,
                              const int64_t* total, uint8_t* out, int64_t cap, int grid, cudaStream_t stream) {
    value_copy_kernel<<<grid, 256, 0, stream>>>(file, pairs, npairs, per_query, stride, kinds, offsets, block_sums,
                                                total, out, cap);
    return cudaGetLastError();
}

}  // namespace gpj
