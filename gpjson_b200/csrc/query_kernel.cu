// find_value: the per-line JSONPath interpreter kernel on sm_100a.
//
// The reference launches find_value once per query with 512x1024 threads
// and a contiguous range of lines per thread
// (functions/QueryFunction.java:201-241, kernels/find_value.cu:12-23).
// Here one launch evaluates every query of the call.  Lines are taken in
// blocks of 32; a block's (line, query) items are nq warps, one query per
// warp and one line per lane, so a warp's lanes follow the same opcode
// sequence and the block's queries run side by side on one SM: the lines'
// bitmap words and key bytes come from DRAM once and are re-read from L1/L2
// by the other queries' warps while still there.  Warps stride over the
// blocks (grid sized to the SMs) and rotate through the queries from one
// block to the next, so a cheap query does not leave its warp idle.  Each
// query writes its own -1-initialised slots, so its results equal a solo run.
#include <cstdint>

#include "interp.cuh"
#include "query_items.cuh"
#include "query_kernel.h"

namespace gpj {

namespace {

// D: level slots of the interpreter's register state (level_slots_for_depth
// of the deepest query of the launch).
template <int D>
__global__ void __launch_bounds__(256) find_value_kernel(QueryParams p) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    LineView view{p.file, p.n, p.string_index, p.leveled, p.level_size, p.n, p.colon};
    const int64_t per_line = 2 * static_cast<int64_t>(p.slots);
    // lines [first, first + lines); the file's last line ends at p.n
    int64_t first = 0, lines = p.num_lines, file_lines = p.num_lines;
    if (p.range) {
        first = p.range[0];
        lines = p.range[1] - first;
        file_lines = p.last ? p.range[1] : INT64_MAX;
    }
    const int64_t items = query_items(lines, p.num_queries);
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < items; g += stride) {
        int64_t li;
        int q;
        if (!query_item(g, 0, lines, p.num_queries, stride, &li, &q)) continue;
        const int64_t i = first + li;
        const bool to_eof = i + 1 >= file_lines;
        if (p.range && (i >= p.out_lines || i + (to_eof ? 0 : 1) >= p.newline_cap)) continue;
        const int64_t start = p.newlines[i];
        const int64_t end = to_eof ? p.n : p.newlines[i + 1];
        int64_t* res = p.out + (static_cast<int64_t>(q) * p.out_lines + i) * per_line;
        run_line<D>(view, start, end, p.bytecode + p.offsets[q], res, per_line);  // writes every slot once
    }
}

template <int D>
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
        int64_t i;
        int q;
        if (!query_item(g - F.item_begin, F.item_begin, F.num_lines, F.num_queries, stride, &i, &q)) continue;
        LineView view{F.file, F.n, F.string_index, F.leveled, F.level_size, F.n, F.colon};
        const int64_t start = F.newlines[i];
        const int64_t end = i + 1 < F.num_lines ? F.newlines[i + 1] : F.n;
        const int64_t per_line = 2 * static_cast<int64_t>(F.slots);
        int64_t* res = F.out + (q * F.out_lines + i) * per_line;
        run_line<D>(view, start, end, F.bytecode + F.offsets[q], res, per_line);
    }
}

}  // namespace

cudaError_t launch_find_value_batch(const QueryFile* files, int nfiles, int64_t total_items, int depth, int grid,
                                    cudaStream_t stream) {
    switch (level_slots_for_depth(depth)) {
        case 5:
            find_value_batch_kernel<5><<<grid, 256, 0, stream>>>(files, nfiles, total_items);
            break;
        case 9:
            find_value_batch_kernel<9><<<grid, 256, 0, stream>>>(files, nfiles, total_items);
            break;
        default:
            find_value_batch_kernel<kLevelSlots><<<grid, 256, 0, stream>>>(files, nfiles, total_items);
    }
    return cudaGetLastError();
}

cudaError_t launch_find_value(const QueryParams& p, int grid, cudaStream_t stream) {
    switch (level_slots_for_depth(p.depth)) {
        case 5:
            find_value_kernel<5><<<grid, 256, 0, stream>>>(p);
            break;
        case 9:
            find_value_kernel<9><<<grid, 256, 0, stream>>>(p);
            break;
        default:
            find_value_kernel<kLevelSlots><<<grid, 256, 0, stream>>>(p);
    }
    return cudaGetLastError();
}

int find_value_max_ctas_per_sm(int depth) {
    int blocks = 0;
    cudaError_t e;
    switch (level_slots_for_depth(depth)) {
        case 5:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, find_value_kernel<5>, 256, 0);
            break;
        case 9:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, find_value_kernel<9>, 256, 0);
            break;
        default:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, find_value_kernel<kLevelSlots>, 256, 0);
    }
    return e == cudaSuccess ? blocks : -1;
}

}  // namespace gpj
