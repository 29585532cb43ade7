// find_value: the per-line JSONPath interpreter kernel on sm_100a.
//
// The reference launches find_value once per query with 512x1024 threads
// and a contiguous range of lines per thread
// (functions/QueryFunction.java:201-241, kernels/find_value.cu:12-23).
// Here one launch evaluates every query of the call: threads stride over
// lines (grid sized to the SMs), and a thread runs all queries on its line
// back to back, so the line's bitmap words and key bytes are fetched from
// DRAM once and re-read from L1/L2 by the following queries.  Each query
// writes its own -1-initialised slots, so its results equal a solo run.
#include <cstdint>

#include "interp.cuh"
#include "query_kernel.h"

namespace gpj {

namespace {

__global__ void __launch_bounds__(256) find_value_kernel(QueryParams p) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    LineView view{p.file, p.n, p.string_index, p.leveled, p.level_size, p.n, nullptr};
    const int64_t lines = p.num_lines;
    const int64_t per_line = 2 * static_cast<int64_t>(p.slots);
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < lines;
         i += stride) {
        const int64_t start = p.newlines[i];
        const int64_t end = i + 1 < lines ? p.newlines[i + 1] : p.n;
        for (int q = 0; q < p.num_queries; q++) {
            int64_t* res = p.out + (static_cast<int64_t>(q) * p.out_lines + i) * per_line;
            for (int64_t k = 0; k < per_line; k++) res[k] = -1;
            run_line(view, start, end, p.bytecode + p.offsets[q], res);
        }
    }
}

__global__ void __launch_bounds__(256) find_value_batch_kernel(const QueryFile* files, int nfiles,
                                                                int64_t total_items) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < total_items; g += stride) {
        int lo = 0, hi = nfiles - 1;  // last file with item_begin <= g
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (files[mid].item_begin <= g)
                lo = mid;
            else
                hi = mid - 1;
        }
        const QueryFile& F = files[lo];
        const int64_t k = g - F.item_begin;
        const int64_t q = k / F.num_lines;
        const int64_t i = k - q * F.num_lines;
        LineView view{F.file, F.n, F.string_index, F.leveled, F.level_size, F.n, nullptr};
        const int64_t start = F.newlines[i];
        const int64_t end = i + 1 < F.num_lines ? F.newlines[i + 1] : F.n;
        const int64_t per_line = 2 * static_cast<int64_t>(F.slots);
        int64_t* res = F.out + (q * F.out_lines + i) * per_line;
        for (int64_t r = 0; r < per_line; r++) res[r] = -1;
        run_line(view, start, end, F.bytecode + F.offsets[q], res);
    }
}

}  // namespace

cudaError_t launch_find_value_batch(const QueryFile* files, int nfiles, int64_t total_items, int grid,
                                    cudaStream_t stream) {
    find_value_batch_kernel<<<grid, 256, 0, stream>>>(files, nfiles, total_items);
    return cudaGetLastError();
}

cudaError_t launch_find_value(const QueryParams& p, int grid, cudaStream_t stream) {
    find_value_kernel<<<grid, 256, 0, stream>>>(p);
    return cudaGetLastError();
}

int find_value_max_ctas_per_sm() {
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, find_value_kernel, 256, 0) != cudaSuccess)
        return -1;
    return blocks;
}

}  // namespace gpj
