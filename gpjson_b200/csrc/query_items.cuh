// Work distribution of the find_value kernels (query_kernel.cu): which
// (line, query) pair a grid-stride item number stands for.  __host__
// __device__ so the test suite can check on the CPU that every pair is
// visited exactly once.
#pragma once

#include <cstdint>

#include "word_ops.cuh"

namespace gpj {

// A file's lines are taken in blocks of 32; block b owns the items
// [item_begin + b * group, item_begin + (b + 1) * group), group = 32 *
// num_queries: one warp per query, one line per lane, so a warp's lanes
// follow one opcode sequence and the block's queries run side by side on
// one SM over the same lines.  The queries of block b are rotated by the
// grid-stride round its first item falls in (the same for all of the
// block's warps), so a warp meets a different query in each round and a
// cheap query does not leave it idle.  `stride` = threads of the grid (a
// multiple of 32); `k` = item number within the file.  Returns false for
// the padding items past the last line.
GPJ_HD bool query_item(int64_t k, int64_t item_begin, int64_t num_lines, int num_queries, int64_t stride,
                       int64_t* line, int* query) {
    const int64_t group = 32 * static_cast<int64_t>(num_queries);
    const int64_t b = k / group;
    const int64_t r = k - b * group;
    *query = static_cast<int>(((r >> 5) + (item_begin + b * group) / stride) % num_queries);
    *line = (b << 5) + (r & 31);
    return *line < num_lines;
}

// Items of a file: ceil(num_lines / 32) blocks of 32 * num_queries (a
// multiple of 32, so no warp spans two files of a batch).
GPJ_HD int64_t query_items(int64_t num_lines, int num_queries) {
    return (num_lines + 31) / 32 * 32 * num_queries;
}

}  // namespace gpj
