// gpj_build_index_device_noalloc: the index build of gpj_build_index_device
// for callers that may not allocate memory (include/gpjson_b200.h).
//
// The kernels are the same two as the context path (line-parallel kernel,
// exact kernel when the input is not well-formed NDJSON); only their scratch
// differs: instead of per-context cudaMalloc'd buffers it is one file-scope
// __device__ array per device, found once with cudaGetSymbolAddress.
//
// Scratch layout (64-bit words):
//   [0, 3 * kMaxTiles)      tile states, tagged with a per-device epoch
//   [kCounterWord]          tile counter, zeroed before every launch
//   [kStatusWord, +2)       status: line count, error bits; zeroed before
//                           every launch
// The tile states must be zero before the first launch and after the 16-bit
// epoch wraps; a zero-initialized __device__ array gives the former, a
// cudaMemsetAsync of the array the latter.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/gpjson_b200.h"
#include "device_common.cuh"
#include "index_kernel.h"

namespace {

constexpr int64_t kMaxBytes = GPJ_NOALLOC_MAX_BYTES;
constexpr int64_t kMaxTiles = kMaxBytes / gpj::kIndexTileBytes;  // 16384
// 3 words per exact-kernel tile also cover the line kernel's 2 per (smaller) tile
static_assert(3 * kMaxTiles >= 2 * ((kMaxBytes + gpj::kLineTileBytes - 1) / gpj::kLineTileBytes),
              "tile states for both kernels");
constexpr int64_t kCounterWord = 3 * kMaxTiles;
constexpr int64_t kStatusWord = kCounterWord + 2;
constexpr int64_t kScratchWords = kStatusWord + 2;  // 49156 words, 384 KiB

static_assert(kMaxBytes % gpj::kIndexTileBytes == 0, "limit must be whole tiles");

__device__ __align__(256) unsigned long long g_scratch[kScratchWords];

constexpr int kMaxDevices = 64;

struct DeviceSetup {
    // held from set-up to the end of a call's device work: calls on one
    // device never overlap on the GPU (they would race on the array)
    std::mutex mu;
    bool ready = false;
    unsigned long long* scratch = nullptr;
    int sms = 0;
    int line_occupancy[3] = {0, 0, 0};   // levels <= 4, <= 8, <= 16
    int exact_occupancy[3] = {0, 0, 0};
    uint32_t epoch = 0;
};

DeviceSetup g_devices[kMaxDevices];

int level_slot(int num_levels) { return num_levels <= 4 ? 0 : (num_levels <= 8 ? 1 : 2); }

// First call on `device` (current): symbol address, SM count, occupancies.
int setup_device(int device, DeviceSetup* d) {
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess) return GPJ_ECUDA;
    if (major != 10) return GPJ_ECUDA;
    if (cudaDeviceGetAttribute(&d->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return GPJ_ECUDA;
    void* addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_scratch) != cudaSuccess || !addr) {
        cudaGetLastError();
        return GPJ_ECUDA;
    }
    d->scratch = static_cast<unsigned long long*>(addr);
    const int levels[3] = {4, 8, 16};
    for (int i = 0; i < 3; i++) {
        d->line_occupancy[i] = gpj::line_index_max_ctas_per_sm(levels[i]);
        d->exact_occupancy[i] = gpj::index_kernel_max_ctas_per_sm(levels[i]);
        if (d->line_occupancy[i] < 1 || d->exact_occupancy[i] < 1) {
            cudaGetLastError();
            return GPJ_ECUDA;
        }
    }
    d->epoch = 0;
    d->ready = true;
    return GPJ_OK;
}

// One launch with the static scratch; h_status receives the status words.
int launch(DeviceSetup* d, bool exact, gpj::IndexParams p, cudaStream_t stream, unsigned long long* h_status) {
    unsigned long long* s = d->scratch;
    if (++d->epoch > 0xFFFFu) {
        if (cudaMemsetAsync(s, 0, 3 * kMaxTiles * sizeof(unsigned long long), stream) != cudaSuccess)
            return GPJ_ECUDA;
        d->epoch = 1;
    }
    if (cudaMemsetAsync(s + kCounterWord, 0, 4 * sizeof(unsigned long long), stream) != cudaSuccess)
        return GPJ_ECUDA;
    p.tile_state = s;
    p.tile_counter = reinterpret_cast<unsigned int*>(s + kCounterWord);
    p.status = s + kStatusWord;
    p.epoch = d->epoch;
    const int slot = level_slot(p.num_levels);
    const int occ = exact ? d->exact_occupancy[slot] : d->line_occupancy[slot];
    int64_t grid = static_cast<int64_t>(d->sms) * occ;
    if (grid > p.ntiles) grid = p.ntiles;
    const cudaError_t e = exact ? gpj::launch_index_kernel(p, static_cast<int>(grid), stream)
                                : gpj::launch_line_index_kernel(p, static_cast<int>(grid), stream);
    if (e != cudaSuccess) return GPJ_ECUDA;
    if (cudaMemcpyAsync(h_status, s + kStatusWord, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                        stream) != cudaSuccess)
        return GPJ_ECUDA;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return GPJ_ECUDA;
    return GPJ_OK;
}

}  // namespace

extern "C" int gpj_build_index_device_noalloc(void* stream_handle, const void* d_file, int64_t n, int num_levels,
                                              uint64_t* d_string_index, uint64_t* d_leveled, int64_t* d_newlines,
                                              int64_t newline_cap, int64_t* num_lines) {
    if (n < 0 || !num_lines || (n > 0 && (!d_file || !d_string_index || !d_leveled)) || newline_cap < 0 ||
        (newline_cap > 0 && !d_newlines))
        return GPJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(d_file) % 16 != 0) return GPJ_EINVAL;
    if (num_levels < 1 || num_levels > GPJ_MAX_LEVELS) return GPJ_ELIMIT;
    if (n > kMaxBytes) return GPJ_ELIMIT;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    // every call reads its status back and waits for its stream, which a
    // stream being captured into a graph does not allow
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &capturing) != cudaSuccess) {
        cudaGetLastError();
        return GPJ_EINVAL;
    }
    if (capturing != cudaStreamCaptureStatusNone) return GPJ_EINVAL;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return GPJ_ECUDA;

    DeviceSetup* d = &g_devices[device];
    std::lock_guard<std::mutex> lock(d->mu);
    if (!d->ready) {
        const int rc = setup_device(device, d);
        if (rc) return rc;
    }
    if (n == 0) {
        if (newline_cap > 0 && cudaMemsetAsync(d_newlines, 0, sizeof(int64_t), stream) != cudaSuccess)
            return GPJ_ECUDA;
        if (cudaStreamSynchronize(stream) != cudaSuccess) return GPJ_ECUDA;
        *num_lines = 1;
        return newline_cap < 1 ? GPJ_ELIMIT : GPJ_OK;
    }
    gpj::IndexParams p{};
    p.file = static_cast<const uint8_t*>(d_file);
    p.n = n;
    p.ntiles = (n + gpj::kIndexTileBytes - 1) / gpj::kIndexTileBytes;
    p.string_index = d_string_index;
    p.leveled = d_leveled;
    p.level_size = (n + 63) / 64;
    p.num_levels = num_levels;
    p.newlines = d_newlines;
    p.newline_cap = newline_cap;
    p.materialize = 1;
    p.tile_begin = 0;
    p.tile_end = p.ntiles;
    p.avail = n;

    gpj::IndexParams lp = p;  // the line-parallel kernel's launch (its own tile size)
    lp.ntiles = (n + gpj::kLineTileBytes - 1) / gpj::kLineTileBytes;
    lp.tile_end = lp.ntiles;

    unsigned long long status[2] = {0, 0};
    int rc = launch(d, false, lp, stream, status);
    if (rc) return rc;
    // a wait that expired in the line pass is reported even when the exact
    // pass that replaces it succeeds
    const unsigned long long line_waits = status[1] & (gpj::kErrLookbackTimeout | gpj::kErrCopyTimeout);
    if (status[1] & (gpj::kErrIrregular | gpj::kErrLongLine)) {
        rc = launch(d, true, p, stream, status);
        if (rc) return rc;
    }
    const unsigned long long errs = (status[1] | line_waits) & ~(gpj::kErrDeferred | gpj::kErrOutOverflow);
    if (errs) return GPJ_EDEVICE;
    *num_lines = static_cast<int64_t>(status[0]);
    return *num_lines > newline_cap ? GPJ_ELIMIT : GPJ_OK;
}
