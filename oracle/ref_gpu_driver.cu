// TEST AND MEASUREMENT INFRASTRUCTURE ONLY: runs the reference's own CUDA
// kernels, compiled from source where they lie in the reference tree (the
// include path is given by oracle/Makefile; nothing is copied), under a
// host driver written here that replays the reference's orchestration:
//   CombinedIndex.create (gpjson/src/main/java/com/koenv/gpjson/stages/
//     CombinedIndex.java:28-151): escape-carry/newline-count kernel, host
//     offsets scan starting at 1, escape + newline index kernel, quote index
//     kernel, host prefix-XOR of the quote carries, string index kernel, all
//     on 8 x 1024 threads;
//   LeveledBitmapsIndex.create (stages/LeveledBitmapsIndex.java:40-103):
//     carry kernel, host level scan starting at -1, leveled bitmaps kernel
//     into zeroed memory;
//   QueryFunction.call (functions/QueryFunction.java:194-241): find_value on
//     512 x 1024 threads per query.
// Differences, both so the outputs can be compared with a solo query: the
// result buffer is reset to -1 before every query (the reference resets it
// once per call and reuses it, QueryFunction.java:194-201), and the buffers
// the reference gets from a fresh cudaMalloc and relies on being zero (the
// escape index, the newline index's entry 0) are zeroed here.  Built with
// -DNDEBUG: the reference kernels' asserts are not compiled in.  The
// reference's counters overflow at 2 GiB (int loop bounds); inputs must be
// smaller.  Only well-formed NDJSON should be given: on other inputs the
// reference kernels can index outside their buffers.
#include <cuda_runtime.h>

#include <cassert>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "create_combined_escape_carry_newline_count_index.cu"
#include "create_combined_escape_newline_index.cu"
#include "create_leveled_bitmaps.cu"
#include "create_leveled_bitmaps_carry_index.cu"
#include "create_quote_index.cu"
#include "create_string_index.cu"
#include "find_value.cu"

namespace {

constexpr int kGrid = 8, kBlock = 1024, kThreads = kGrid * kBlock;

#define REF_CHECK(x)                              \
    do {                                          \
        cudaError_t e_ = (x);                     \
        if (e_ != cudaSuccess) return -static_cast<int>(e_) - 1000; \
    } while (0)

struct Buffers {
    char* file = nullptr;
    char* carry = nullptr;       // escape carry, then quote carry (int8 per thread)
    int* counts = nullptr;       // newline counts, then offsets
    long* escape = nullptr;
    long* string = nullptr;      // quote index, then string index
    long* newlines = nullptr;
    long* leveled = nullptr;
    char* level_carry = nullptr;
    char* query = nullptr;
    long* result = nullptr;
    void release() {
        for (void* p : {static_cast<void*>(file), static_cast<void*>(carry), static_cast<void*>(counts),
                        static_cast<void*>(escape), static_cast<void*>(string), static_cast<void*>(newlines),
                        static_cast<void*>(leveled), static_cast<void*>(level_carry), static_cast<void*>(query),
                        static_cast<void*>(result)})
            if (p) cudaFree(p);
    }
};

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// CombinedIndex.create + LeveledBitmapsIndex.create; *lines = newline index size.
int build_index(Buffers& b, int64_t n, int num_levels, int64_t* lines) {
    const int64_t words = (n + 63) / 64;
    create_combined_escape_carry_newline_count_index<<<kGrid, kBlock>>>(b.file, n, b.carry, b.counts);
    REF_CHECK(cudaGetLastError());
    std::vector<int> counts(kThreads);
    REF_CHECK(cudaMemcpy(counts.data(), b.counts, sizeof(int) * kThreads, cudaMemcpyDeviceToHost));
    int sum = 1;  // CombinedIndex.createOffsetsIndex: the first "newline" is position 0
    for (int i = 0; i < kThreads; i++) {
        const int v = counts[i];
        counts[i] = sum;
        sum += v;
    }
    REF_CHECK(cudaMemcpy(b.counts, counts.data(), sizeof(int) * kThreads, cudaMemcpyHostToDevice));
    if (b.newlines) cudaFree(b.newlines);
    b.newlines = nullptr;
    REF_CHECK(cudaMalloc(&b.newlines, sizeof(long) * sum));
    REF_CHECK(cudaMemset(b.newlines, 0, sizeof(long) * sum));
    REF_CHECK(cudaMemset(b.escape, 0, sizeof(long) * words));
    create_combined_escape_newline_index<<<kGrid, kBlock>>>(b.file, n, reinterpret_cast<bool*>(b.carry), b.counts,
                                                            b.escape, words, b.newlines);
    REF_CHECK(cudaGetLastError());
    create_quote_index<<<kGrid, kBlock>>>(b.file, n, b.escape, b.string, b.carry, words);
    REF_CHECK(cudaGetLastError());
    std::vector<signed char> carry(kThreads);
    REF_CHECK(cudaMemcpy(carry.data(), b.carry, kThreads, cudaMemcpyDeviceToHost));
    signed char prev = 0;  // CombinedIndex.createQuoteIndex: prefix XOR of the carries
    for (int i = 0; i < kThreads; i++) {
        prev = static_cast<signed char>(carry[i] ^ prev);
        carry[i] = prev;
    }
    REF_CHECK(cudaMemcpy(b.carry, carry.data(), kThreads, cudaMemcpyHostToDevice));
    create_string_index<<<kGrid, kBlock>>>(words, b.string, b.carry);
    REF_CHECK(cudaGetLastError());
    // LeveledBitmapsIndex.create
    REF_CHECK(cudaMemset(b.leveled, 0, sizeof(long) * words * num_levels));
    create_leveled_bitmaps_carry_index<<<kGrid, kBlock>>>(b.file, n, b.string, b.level_carry);
    REF_CHECK(cudaGetLastError());
    std::vector<signed char> levels(kThreads);
    REF_CHECK(cudaMemcpy(levels.data(), b.level_carry, kThreads, cudaMemcpyDeviceToHost));
    signed char level = -1;  // LeveledBitmapsIndex.createLevelsIndex
    for (int i = 0; i < kThreads; i++) {
        const signed char v = levels[i];
        levels[i] = level;
        level = static_cast<signed char>(level + v);
    }
    REF_CHECK(cudaMemcpy(b.level_carry, levels.data(), kThreads, cudaMemcpyHostToDevice));
    create_leveled_bitmaps<<<kGrid, kBlock>>>(b.file, n, b.string, b.level_carry, b.leveled, words * num_levels,
                                              words, num_levels);
    REF_CHECK(cudaGetLastError());
    REF_CHECK(cudaDeviceSynchronize());
    *lines = sum;
    return 0;
}

}  // namespace

extern "C" {

// Index and queries of `n` host bytes with the reference kernels, `repeats`
// times on the device-resident input (after one untimed round).  Outputs of
// the last round go to the host buffers given (each may be null): string
// index (ceil(n/64) words), leveled bitmaps (num_levels x words), newline
// index (nl_cap entries), results int64[nq][lines][slots][2] (res_cap
// elements).  *index_ms / *query_ms: mean wall time of a round's index
// build (kernels and the reference's host scans and copies) and of its nq
// find_value launches (with the per-query reset).  Returns 0, -1 for bad
// arguments or too small buffers (*lines still set), or -1000 - a CUDA error.
__attribute__((visibility("default"))) int ref_gpu_run(const uint8_t* host, int64_t n, int num_levels, int nq,
                                                       const uint8_t* const* bytecode, const size_t* lengths,
                                                       int slots, int repeats, uint64_t* h_string,
                                                       uint64_t* h_leveled, int64_t* h_newlines, int64_t nl_cap,
                                                       int64_t* lines, int64_t* h_results, int64_t res_cap,
                                                       double* index_ms, double* query_ms) {
    if (!host || n <= 0 || n >= (1ll << 31) || num_levels < 1 || num_levels > 16 || nq < 1 || slots < 1 ||
        repeats < 1 || !lines || !index_ms || !query_ms)
        return -1;
    const int64_t words = (n + 63) / 64;
    size_t max_query = 0;
    for (int q = 0; q < nq; q++) max_query = lengths[q] > max_query ? lengths[q] : max_query;
    Buffers b;
    auto run = [&]() -> int {
        REF_CHECK(cudaMalloc(&b.file, n));
        REF_CHECK(cudaMemcpy(b.file, host, n, cudaMemcpyHostToDevice));
        REF_CHECK(cudaMalloc(&b.carry, kThreads));
        REF_CHECK(cudaMalloc(&b.counts, sizeof(int) * kThreads));
        REF_CHECK(cudaMalloc(&b.escape, sizeof(long) * words));
        REF_CHECK(cudaMalloc(&b.string, sizeof(long) * words));
        REF_CHECK(cudaMemset(b.string, 0, sizeof(long) * words));
        REF_CHECK(cudaMalloc(&b.leveled, sizeof(long) * words * num_levels));
        REF_CHECK(cudaMalloc(&b.level_carry, kThreads));
        REF_CHECK(cudaMalloc(&b.query, max_query));
        double t_index = 0, t_query = 0;
        int64_t count = 0;
        auto queries = [&](int64_t* out) -> int {
            for (int q = 0; q < nq; q++) {
                REF_CHECK(cudaMemcpy(b.query, bytecode[q], lengths[q], cudaMemcpyHostToDevice));
                REF_CHECK(cudaMemset(b.result, 0xFF, sizeof(long) * count * 2 * slots));
                find_value<<<512, 1024>>>(b.file, n, b.newlines, count, b.string, b.leveled, words * num_levels, words,
                                          b.query, slots, b.result);
                REF_CHECK(cudaGetLastError());
                if (out)
                    REF_CHECK(cudaMemcpy(out + static_cast<int64_t>(q) * count * 2 * slots, b.result,
                                         sizeof(long) * count * 2 * slots, cudaMemcpyDeviceToHost));
            }
            REF_CHECK(cudaDeviceSynchronize());
            return 0;
        };
        for (int r = 0; r <= repeats; r++) {  // repeat 0 untimed (warm-up)
            const double t0 = now_ms();
            int rc = build_index(b, n, num_levels, &count);
            if (rc) return rc;
            const double t1 = now_ms();
            if (!b.result) REF_CHECK(cudaMalloc(&b.result, sizeof(long) * count * 2 * slots));
            rc = queries(nullptr);
            if (rc) return rc;
            const double t2 = now_ms();
            if (r > 0) {
                t_index += t1 - t0;
                t_query += t2 - t1;
            }
        }
        if (h_results) {  // once more, untimed, copying each query's results
            if (res_cap < static_cast<int64_t>(nq) * count * 2 * slots) {
                *lines = count;
                return -1;
            }
            int rc = queries(h_results);
            if (rc) return rc;
        }
        *index_ms = t_index / repeats;
        *query_ms = t_query / repeats;
        *lines = count;
        if (h_string) REF_CHECK(cudaMemcpy(h_string, b.string, sizeof(long) * words, cudaMemcpyDeviceToHost));
        if (h_leveled)
            REF_CHECK(cudaMemcpy(h_leveled, b.leveled, sizeof(long) * words * num_levels, cudaMemcpyDeviceToHost));
        if (h_newlines) {
            if (nl_cap < count) return -1;
            REF_CHECK(cudaMemcpy(h_newlines, b.newlines, sizeof(long) * count, cudaMemcpyDeviceToHost));
        }
        return 0;
    };
    const int rc = run();
    b.release();
    return rc;
}

}  // extern "C"
