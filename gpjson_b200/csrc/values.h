// Host-side interface of the value-extraction kernels (values.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace gpj {

// Kinds of a result pair (start, end): null (start == -1), a value
// file[start, end), or unreadable (end before start: the reference's
// ResultItem fails to build such a value).
constexpr uint8_t kValueNull = 0;
constexpr uint8_t kValuePresent = 1;
constexpr uint8_t kValueUnreadable = 2;

// Scratch entries (int64) launch_value_sizes needs for npairs pairs.
int64_t value_scan_blocks(int64_t npairs);

// Pass 1: kinds[npairs], block-local offsets, and the byte total into
// device memory `total` (block_sums: value_scan_blocks(npairs) entries).
// Pair i = q * per_query + r is read at pairs[2 * (q * stride + r)]; n is
// the file size (pairs reaching past it are unreadable).
cudaError_t launch_value_sizes(const int64_t* pairs, int64_t npairs, int64_t per_query, int64_t stride, int64_t n,
                               uint8_t* kinds, int64_t* offsets, int64_t* block_sums, int64_t* total,
                               cudaStream_t stream);

// Pass 2: offsets[0..npairs] final (offsets[npairs] = total) and each
// value's bytes at out[offsets[i]] (values ending past `cap` are skipped).
cudaError_t launch_value_copy(const uint8_t* file, const int64_t* pairs, int64_t npairs, int64_t per_query,
                              int64_t stride, const uint8_t* kinds, int64_t* offsets, const int64_t* block_sums,
                              const int64_t* total, uint8_t* out, int64_t cap, int grid, cudaStream_t stream);

}  // namespace gpj
