// Host-side interface of the find_value kernel (query_kernel.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "query_items.cuh"

namespace gpj {

// A (line, query) item handed from the thread-per-line kernels to the
// warp-per-line kernel (line of file `file` of the launch).
struct LongItem {
    int64_t line;
    int32_t file;
    int32_t query;
};

// Where the thread-per-line kernels put lines longer than `bytes`, which a
// whole warp then evaluates (find_value_long): `items` holds `cap` entries,
// `count` (zeroed before the launch) counts them; items past `cap` are
// evaluated by their thread.  items == nullptr: no line is handed over.
struct LongLines {
    LongItem* items;
    unsigned long long* count;
    int64_t cap;
    int64_t bytes;
};

// Threads per CTA of find_value_kernel and find_value_batch_kernel (a
// multiple of 32; grids are sized in these CTAs), and the CTAs per SM their
// register budget is set for, by register-state size D: 7 (at most 72
// registers) for D = 5, 6 for D = 9, 4 for D = 17.  128-thread CTAs at 72
// registers keep 28 warps per SM resident where 256-thread CTAs at 80 kept 24.
constexpr int kQueryThreads = 128;
template <int D>
constexpr int kQueryMinCtas = D <= 5 ? 7 : (D <= 9 ? 6 : 4);

struct QueryParams {
    const uint8_t* file;
    int64_t n;
    const int64_t* newlines;
    int64_t num_lines;
    const uint64_t* string_index;
    const uint64_t* leveled;
    int64_t level_size;
    const uint8_t* bytecode;  // all queries back to back
    const int32_t* offsets;   // start of query q in `bytecode`
    int num_queries;
    int slots;     // result slots per line (max num_results)
    int64_t* out;       // [num_queries][out_lines][slots][2]
    int64_t out_lines;  // query stride of `out` (>= num_lines)
    // Optional, for a file still being indexed: only lines [range[0],
    // range[1]) (device memory, read by the kernel), whose newline-index
    // entries up to range[1] are written; the last of them ends at the file
    // end when `last`, else at newlines[range[1]].  Lines whose results or
    // end do not fit out_lines / newline_cap are skipped (the caller sees the
    // line count and evaluates again).
    const int64_t* range;
    int last;
    int64_t newline_cap;
    // Optional ':' outside strings (level_size words): key searches jump
    // between structural colons, index searches between the other
    // structural bytes (the bytes each search ignores).
    const uint64_t* colon;
    // deepest level of the launch's queries (sizes the interpreter's
    // register state)
    int depth;
    LongLines long_lines;
};

// find_value over the launch's lines, then (when p.long_lines.items is set)
// the long lines a warp each, with `long_grid` CTAs.
cudaError_t launch_find_value(const QueryParams& p, int grid, int long_grid, cudaStream_t stream);
// Resident CTAs per SM of the find_value kernel for queries of that depth.
int find_value_max_ctas_per_sm(int depth);

// One file of a batched find_value launch: its index, its queries and where
// their results go ([num_queries][out_lines][slots][2]); its lines are
// [line_begin, line_begin + num_lines) of the batch's line numbering.
struct QueryFile {
    const uint8_t* file;
    int64_t n;
    const int64_t* newlines;
    int64_t num_lines;
    const uint64_t* string_index;
    const uint64_t* leveled;
    int64_t level_size;
    const uint8_t* bytecode;
    const int32_t* offsets;
    int num_queries;
    int slots;
    int64_t* out;
    int64_t out_lines;
    // first of the file's items in the batch: ceil(num_lines / 32) blocks of
    // 32 lines x num_queries (a multiple of 32, so no warp spans two files)
    int64_t item_begin;
    const uint64_t* colon;  // optional, as QueryParams::colon
};

// Every (line, query) item of every file of the batch (`files`: device
// array, ascending item_begin, total_items items in all; `depth` the deepest
// level of any of their queries), one per thread:
// a warp's lanes run one query on 32 lines of one file, and the warps of a
// block of lines run its queries side by side.
cudaError_t launch_find_value_batch(const QueryFile* files, int nfiles, int64_t total_items, int depth,
                                    const LongLines& long_lines, int grid, int long_grid, cudaStream_t stream);

}  // namespace gpj
