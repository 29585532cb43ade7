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

// The scans of one line by the 32 lanes of a warp together (all lanes call
// with the same arguments and hold the same interpreter state): a search
// for the next structural bit reads 32 bitmap words per step, a whitespace
// skip 512 bytes, so a line of a megabyte costs its warp a few hundred
// dependent memory round trips instead of one lane tens of thousands.
struct WarpScan {
    template <typename P>
    __device__ static P next_masked(const uint64_t* bm, const uint64_t* filt, uint64_t flip, P from, P limit, P& cw,
                                    uint64_t& cv) {
        if (from >= limit) return limit;
        const int lane = threadIdx.x & 31;
        const P w = from >> 6;
        const P wend = ((limit - 1) >> 6) + 1;
        const uint64_t first = w == cw ? cv : (bm[w] & (filt ? (filt[w] ^ flip) : ~0ull));
        const uint64_t m = first & (~0ull << (from & 63));
        if (m) {
            cw = w;
            cv = first;
            const P p = (w << 6) + ctz64(m);
            return p < limit ? p : limit;
        }
        for (P b = w + 1; b < wend; b += 32) {
            const P wl = b + lane;
            const uint64_t x = wl < wend ? (bm[wl] & (filt ? (filt[wl] ^ flip) : ~0ull)) : 0ull;
            const unsigned hit = __ballot_sync(~0u, x != 0);
            if (hit) {
                const int f = __ffs(static_cast<int>(hit)) - 1;
                cw = b + f;
                cv = __shfl_sync(~0u, x, f);
                const P p = (cw << 6) + ctz64(cv);
                return p < limit ? p : limit;
            }
        }
        return limit;
    }
    template <typename P>
    __device__ static P next(const uint64_t* bm, P from, P limit, P& cw, uint64_t& cv) {
        return next_masked<P>(bm, nullptr, 0ull, from, limit, cw, cv);
    }
    template <typename P>
    __device__ static P next_filtered(const uint64_t* bm, const uint64_t* filt, bool invert, P from, P limit, P& cw,
                                      uint64_t& cv) {
        return next_masked<P>(bm, filt, invert ? ~0ull : 0ull, from, limit, cw, cv);
    }
    // first position at or after j that is >= hi or not whitespace
    template <typename P>
    __device__ static P skip(const uint8_t* file, P j, P hi) {
        const int lane = threadIdx.x & 31;
        for (int k = 0; k < 32; k++, ++j)
            if (j >= hi || !is_ws(file[j])) return j;
        for (; j < hi && (reinterpret_cast<uintptr_t>(file + j) & 15) != 0; ++j)
            if (!is_ws(file[j])) return j;
        for (;; j += 512) {
            const P q = j + 16 * lane;
            P stop = -1;  // this lane's answer among its 16 bytes, if any
            if (q + 16 <= hi) {
                const uint4 v = *reinterpret_cast<const uint4*>(file + q);
                if (!(all_ws32(v.x) && all_ws32(v.y) && all_ws32(v.z) && all_ws32(v.w))) {
                    for (int b = 0; b < 16; b++) {
                        if (!is_ws(file[q + b])) {
                            stop = q + b;
                            break;
                        }
                    }
                }
            } else {
                for (int b = 0; b < 16; b++) {
                    const P r = q + b;
                    if (r >= hi || !is_ws(file[r])) {
                        stop = r;
                        break;
                    }
                }
            }
            const unsigned hit = __ballot_sync(~0u, stop >= 0);
            if (hit) return __shfl_sync(~0u, stop, __ffs(static_cast<int>(hit)) - 1);
        }
    }
    __device__ static void store(int64_t* res, int64_t k, int64_t v) {
        if ((threadIdx.x & 31) == 0) res[k] = v;
    }
};

// Hands item (line, file, query) to the warp-per-line kernel; false when the
// list is full (the caller evaluates it).
__device__ __forceinline__ bool hand_over(const LongLines& L, int64_t line, int file, int query) {
    const unsigned long long slot = atomicAdd(L.count, 1ull);
    if (static_cast<int64_t>(slot) >= L.cap) return false;
    L.items[slot] = LongItem{line, file, query};
    return true;
}

// One long line on a whole warp: the interpreter in 64-bit positions, every
// lane in the same state, lane 0 writing the results.
template <int D>
__device__ __forceinline__ void run_long_line(const LineView& view, int64_t start, int64_t end, const uint8_t* ir,
                                              int64_t* res, int64_t per_line) {
    RegLevelsT<D, int64_t> lv;
    int stored = 0;
    run_line_core<int64_t, RegLevelsT<D, int64_t>, WarpScan>(view.file, view.n, view.n, kLineDone, view.string_index,
                                                             view.levels, view.level_size, view.colon, start, end, ir,
                                                             res, 0, lv, stored);
    if ((threadIdx.x & 31) == 0)
        for (int64_t k = 2 * static_cast<int64_t>(stored); k < per_line; k++) res[k] = -1;
}

// D: level slots of the interpreter's register state (level_slots_for_depth
// of the deepest query of the launch).
template <int D>
__global__ void __launch_bounds__(kQueryThreads, kQueryMinCtas<D>) find_value_kernel(QueryParams p) {
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
        if (p.long_lines.items && end - start > p.long_lines.bytes && hand_over(p.long_lines, i, 0, q)) continue;
        int64_t* res = p.out + (static_cast<int64_t>(q) * p.out_lines + i) * per_line;
        const uint8_t* ir = p.bytecode + p.offsets[q];
        // writes every slot once, unless a whitespace skip runs far past the
        // line (then a warp evaluates it again)
        if (run_line<D>(view, start, end, ir, res, per_line, kRelLimit,
                        p.long_lines.items ? p.long_lines.bytes : -1) == kLineLong &&
            !hand_over(p.long_lines, i, 0, q))
            run_line_wide(view, start, end, ir, res, per_line);
    }
}

// The lines find_value_kernel handed over, a warp each.
template <int D>
__global__ void __launch_bounds__(256) find_value_long_kernel(QueryParams p) {
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    const int64_t count = *p.long_lines.count < static_cast<unsigned long long>(p.long_lines.cap)
                              ? static_cast<int64_t>(*p.long_lines.count)
                              : p.long_lines.cap;
    LineView view{p.file, p.n, p.string_index, p.leveled, p.level_size, p.n, p.colon};
    const int64_t per_line = 2 * static_cast<int64_t>(p.slots);
    const int64_t file_lines = p.range ? (p.last ? p.range[1] : INT64_MAX) : p.num_lines;
    for (int64_t k = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; k < count; k += warps) {
        const LongItem it = p.long_lines.items[k];
        const int64_t i = it.line;
        const int64_t start = p.newlines[i];
        const int64_t end = i + 1 >= file_lines ? p.n : p.newlines[i + 1];
        int64_t* res = p.out + (static_cast<int64_t>(it.query) * p.out_lines + i) * per_line;
        run_long_line<D>(view, start, end, p.bytecode + p.offsets[it.query], res, per_line);
    }
}

template <int D>
__global__ void __launch_bounds__(kQueryThreads, kQueryMinCtas<D>) find_value_batch_kernel(const QueryFile* files, int nfiles,
                                                                int64_t total_items, LongLines long_lines) {
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
        if (long_lines.items && end - start > long_lines.bytes && hand_over(long_lines, i, lo, q)) continue;
        const int64_t per_line = 2 * static_cast<int64_t>(F.slots);
        int64_t* res = F.out + (q * F.out_lines + i) * per_line;
        const uint8_t* ir = F.bytecode + F.offsets[q];
        if (run_line<D>(view, start, end, ir, res, per_line, kRelLimit, long_lines.items ? long_lines.bytes : -1) ==
                kLineLong &&
            !hand_over(long_lines, i, lo, q))
            run_line_wide(view, start, end, ir, res, per_line);
    }
}

template <int D>
__global__ void __launch_bounds__(256) find_value_batch_long_kernel(const QueryFile* files, LongLines long_lines) {
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    const int64_t count = *long_lines.count < static_cast<unsigned long long>(long_lines.cap)
                              ? static_cast<int64_t>(*long_lines.count)
                              : long_lines.cap;
    for (int64_t k = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; k < count; k += warps) {
        const LongItem it = long_lines.items[k];
        const QueryFile& F = files[it.file];
        LineView view{F.file, F.n, F.string_index, F.leveled, F.level_size, F.n, F.colon};
        const int64_t i = it.line;
        const int64_t start = F.newlines[i];
        const int64_t end = i + 1 < F.num_lines ? F.newlines[i + 1] : F.n;
        const int64_t per_line = 2 * static_cast<int64_t>(F.slots);
        int64_t* res = F.out + (it.query * F.out_lines + i) * per_line;
        run_long_line<D>(view, start, end, F.bytecode + F.offsets[it.query], res, per_line);
    }
}

template <int D>
cudaError_t launch_batch_d(const QueryFile* files, int nfiles, int64_t total_items, const LongLines& L, int grid,
                           int long_grid, cudaStream_t stream) {
    find_value_batch_kernel<D><<<grid, kQueryThreads, 0, stream>>>(files, nfiles, total_items, L);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && L.items) {
        find_value_batch_long_kernel<D><<<long_grid, 256, 0, stream>>>(files, L);
        e = cudaGetLastError();
    }
    return e;
}

template <int D>
cudaError_t launch_d(const QueryParams& p, int grid, int long_grid, cudaStream_t stream) {
    find_value_kernel<D><<<grid, kQueryThreads, 0, stream>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && p.long_lines.items) {
        find_value_long_kernel<D><<<long_grid, 256, 0, stream>>>(p);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace

cudaError_t launch_find_value_batch(const QueryFile* files, int nfiles, int64_t total_items, int depth,
                                    const LongLines& long_lines, int grid, int long_grid, cudaStream_t stream) {
    switch (level_slots_for_depth(depth)) {
        case 5:
            return launch_batch_d<5>(files, nfiles, total_items, long_lines, grid, long_grid, stream);
        case 9:
            return launch_batch_d<9>(files, nfiles, total_items, long_lines, grid, long_grid, stream);
        default:
            return launch_batch_d<kLevelSlots>(files, nfiles, total_items, long_lines, grid, long_grid, stream);
    }
}

cudaError_t launch_find_value(const QueryParams& p, int grid, int long_grid, cudaStream_t stream) {
    switch (level_slots_for_depth(p.depth)) {
        case 5:
            return launch_d<5>(p, grid, long_grid, stream);
        case 9:
            return launch_d<9>(p, grid, long_grid, stream);
        default:
            return launch_d<kLevelSlots>(p, grid, long_grid, stream);
    }
}

int find_value_max_ctas_per_sm(int depth) {
    int blocks = 0;
    cudaError_t e;
    switch (level_slots_for_depth(depth)) {
        case 5:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, find_value_kernel<5>, kQueryThreads, 0);
            break;
        case 9:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, find_value_kernel<9>, kQueryThreads, 0);
            break;
        default:
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, find_value_kernel<kLevelSlots>, kQueryThreads, 0);
    }
    return e == cudaSuccess ? blocks : -1;
}

}  // namespace gpj
