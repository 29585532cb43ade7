// C ABI of gpjson_b200 (include/gpjson_b200.h): contexts, input files,
// index builds, queries, results and diagnostics.
//
// This is the host runtime that replaces the reference's grCUDA-derived
// CUDARuntime (gpu/CUDARuntime.java) and the orchestration of
// functions/QueryFunction.java:48-265 and the stages/ classes.
#include <cuda_runtime.h>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gpjson_b200.h"
#include "device_common.cuh"
#include "host_io.h"
#include "index_kernel.h"
#include "jsonpath.h"
#include "query_kernel.h"
#include "values.h"

namespace {

thread_local std::string g_create_error;

struct Phase {
    std::string name;
    double device_ms;  // CUDA-event time on the context's stream
    double host_ms;    // wall time of the call around it
};

}  // namespace

// Longest run past a tile the batched index launch follows to finish a line.
static constexpr int64_t kBatchMaxExtension = 8ll << 20;

// Entries of a context's list of long lines handed to a warp each.
static constexpr int64_t kLongItems = 1 << 16;

static gpj_tuning default_tuning() {
    gpj_tuning t{};
    t.long_line_bytes = 65536;
    t.query_ctas_per_sm = 0;
    t.index_ctas_per_sm = 0;
    t.chunk_tiles = 0;
    return t;
}

struct gpj_ctx {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // host-to-device copies overlapped with indexing
    // Device buffers come from this stream-ordered pool; freed blocks stay
    // reserved for the next file instead of going back to the driver.
    cudaMemPool_t pool = nullptr;
    std::vector<cudaEvent_t> chunk_events;  // one per loaded chunk
    cudaEvent_t ev_ready = nullptr;
    std::string err;

    // scratch of the index kernel
    unsigned long long* d_tile_state = nullptr;
    int64_t tile_state_words = 0;
    unsigned int* d_counter = nullptr;
    unsigned long long* d_status = nullptr;
    unsigned long long* h_status = nullptr;  // pinned, 2 words
    uint32_t epoch = 0;
    int index_occupancy[3] = {0, 0, 0};  // exact kernel, levels <=4, <=8, <=16
    int line_occupancy[3] = {0, 0, 0};   // line-parallel kernel
    int tile_occupancy[3] = {0, 0, 0};   // its standalone form (index builds without queries)
    int64_t exact_fallbacks = 0;         // builds that needed the exact kernel
    bool fuse_queries = false;           // evaluate queries inside the index kernel
    unsigned path_extensions = 0;        // GPJ_PATH_* flags for calls that compile paths
    int query_occupancy[3] = {0, 0, 0};  // find_value CTAs per SM, by register-state size (depth <= 4, <= 8, more)
    // lines find_value hands to a warp each (gpj_tuning); the hand-over list
    gpj_tuning tuning{};
    gpj::LongItem* d_long = nullptr;
    unsigned long long* d_long_count = nullptr;

    // pinned staging for file reads
    uint8_t* h_stage = nullptr;
    size_t stage_bytes = 0;

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t launches = 0;
    std::vector<Phase> phases;
};

struct gpj_file {
    gpj_ctx* ctx = nullptr;
    const uint8_t* d_data = nullptr;
    uint8_t* d_owned = nullptr;
    int64_t n = 0;
    int64_t words = 0;

    uint64_t* d_str = nullptr;
    uint64_t* d_colon = nullptr;  // ':' outside strings, for find_value's key searches
    bool colon_valid = false;     // d_colon belongs to the current index
    uint64_t* d_lvl = nullptr;
    int lvl_cap = 0;
    int64_t* d_nl = nullptr;
    int64_t nl_cap = 0;
    bool indexed = false;
    bool exact_only = false;  // the line kernels flagged this input: index it with the exact kernel
    int num_levels = 0;
    int64_t num_lines = 0;

    // uploaded bytecode (cached across calls with identical queries)
    std::vector<uint8_t> ir_host;
    int ir_depth = 0;  // deepest level of the uploaded queries
    uint8_t* d_ir = nullptr;
    size_t d_ir_cap = 0;
    // results of gpj_query with a host destination
    int64_t* d_out = nullptr;
    size_t d_out_cap = 0;  // elements
};

// The page-locked results of one batch run, shared by the batch and the
// gpj_result views handed out for it (gpj_batch_result_ex); the last owner
// frees it.
struct PinnedResults {
    int64_t* p = nullptr;
    size_t cap = 0;  // elements
    std::atomic<int> refs{1};
};

static void unref(PinnedResults* r) {
    if (r && r->refs.fetch_sub(1) == 1) {
        cudaFreeHost(r->p);
        delete r;
    }
}

struct gpj_result {
    int64_t nq = 0, lines = 0;
    int slots = 0;
    // [nq][lines][slots][2], copied in, or inside `backing`
    int64_t* offsets = nullptr;
    size_t cap = 0;  // elements of `offsets` (when not a view)
    PinnedResults* backing = nullptr;

    gpj_result() = default;
    gpj_result(const gpj_result&) = delete;
    gpj_result& operator=(const gpj_result&) = delete;
    ~gpj_result() {
        if (backing)
            unref(backing);
        else
            gpj::result_buffers().give(offsets, cap);
    }

    bool allocate(size_t count) {
        offsets = gpj::result_buffers().take(std::max<size_t>(count, 1), &cap);
        return offsets != nullptr;
    }
};

// Values of a query call gathered on the device (gpj_query_values).
struct gpj_values {
    int64_t nq = 0, lines = 0;
    int slots = 0;
    std::vector<uint8_t> kinds;     // [nq][lines][slots]
    std::vector<int64_t> offsets;   // [nq * lines * slots + 1]
    std::vector<uint8_t> bytes;     // offsets.back() bytes
};

// Requests (file, paths) evaluated together by gpj_batch_run.
struct gpj_batch {
    gpj_ctx* ctx = nullptr;
    struct Item {
        gpj_file* file = nullptr;
        std::vector<gpj::CompiledPath> queries;
        int file_slot = -1;  // index into `files` after a run
        int q0 = 0;          // first of the item's queries in its file's query list
    };
    struct FileRun {
        gpj_file* file = nullptr;
        std::vector<const gpj::CompiledPath*> queries;
        int depth = 0, slots = 1;
        int64_t lines = 0;
        size_t out_offset = 0;  // elements into `results`
    };
    std::vector<Item> items;
    std::vector<FileRun> files;
    // results of the last run, page-locked (one copy from the device at full
    // speed); buffers no result refers to any more are used again
    std::vector<PinnedResults*> pool;
    PinnedResults* cur = nullptr;
    bool ran = false;
    // The query phase of the last run as a CUDA graph (find_value over every
    // item, the long-line warps, the copy of the results), replayed by the
    // next run when neither the requests nor the files' indexes nor the
    // launch shapes changed and no result of the last run is still held.
    struct Replay {
        cudaGraphExec_t exec = nullptr;
        std::vector<uint64_t> sig;  // what the graph reads (files' buffers, line counts, tuning)
        uint8_t* d_blob = nullptr;  // kept while the graph lives
        int64_t* d_out = nullptr;
        gpj::QueryFile* d_qf = nullptr;
        PinnedResults* dst = nullptr;  // the copy's destination
        cudaStream_t stream = nullptr;
    } replay;
    bool dirty = true;  // requests added or cleared since the graph was made
    int64_t replays = 0;
    ~gpj_batch() {
        drop_replay();
        for (PinnedResults* r : pool) unref(r);
    }
    void drop_replay() {
        if (replay.exec) cudaGraphExecDestroy(replay.exec);
        // pool allocations of the batch's context, freed in its stream order
        if (replay.d_blob) cudaFreeAsync(replay.d_blob, replay.stream);
        if (replay.d_out) cudaFreeAsync(replay.d_out, replay.stream);
        if (replay.d_qf) cudaFreeAsync(replay.d_qf, replay.stream);
        replay = Replay{};
    }
};

namespace {

int fail(gpj_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(gpj_ctx* ctx, cudaError_t e, const char* what) {
    char buf[256];
    std::snprintf(buf, sizeof buf, "CUDA error %d (%s: %s) in %s", static_cast<int>(e),
                  cudaGetErrorName(e), cudaGetErrorString(e), what);
    return fail(ctx, e == cudaErrorMemoryAllocation ? GPJ_ENOMEM : GPJ_ECUDA, buf);
}

#define GPJ_CUDA(ctx, call)                                        \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call); \
    } while (0)

// Stream-ordered allocation from the context's pool on the context's stream
// (other streams that touch the buffer wait for an event recorded after it).
template <typename T>
int device_alloc(gpj_ctx* ctx, T** p, size_t count, const char* what) {
    void* q = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&q, std::max<size_t>(count * sizeof(T), 16), ctx->pool, ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(ctx, e, what);
    }
    *p = static_cast<T*>(q);
    return GPJ_OK;
}

template <typename T>
void device_free(gpj_ctx* ctx, T*& p) {
    if (p) cudaFreeAsync(p, ctx->stream);
    p = nullptr;
}

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Records a phase measured between ev0 (recorded at `host_start`) and now.
int end_phase(gpj_ctx* ctx, const char* name, double host_start) {
    GPJ_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    GPJ_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    GPJ_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->phases.push_back(Phase{name, static_cast<double>(ms), now_ms() - host_start});
    return GPJ_OK;
}

int ensure_tile_state(gpj_ctx* ctx, int64_t ntiles) {
    const int64_t words = 3 * ntiles;
    if (words > ctx->tile_state_words) {
        device_free(ctx, ctx->d_tile_state);
        ctx->tile_state_words = 0;
        const int64_t cap = std::max<int64_t>(words, 3 * 4096);
        int rc = device_alloc(ctx, &ctx->d_tile_state, static_cast<size_t>(cap), "cudaMalloc(tile state)");
        if (rc) return rc;
        GPJ_CUDA(ctx, cudaMemsetAsync(ctx->d_tile_state, 0, cap * 8, ctx->stream));
        ctx->tile_state_words = cap;
        ctx->epoch = 0;
    }
    if (++ctx->epoch > 0xFFFFu) {  // tags wrapped: clear and restart
        GPJ_CUDA(ctx, cudaMemsetAsync(ctx->d_tile_state, 0, ctx->tile_state_words * 8, ctx->stream));
        ctx->epoch = 1;
    }
    return GPJ_OK;
}

int occupancy_slot(int num_levels) { return num_levels <= 4 ? 0 : (num_levels <= 8 ? 1 : 2); }

// The standalone index kernel's tile counter (the second word of d_counter;
// the exact kernel uses the first).
unsigned int* tile_claims(gpj_ctx* ctx) { return ctx->d_counter + 1; }

// One launch of an index kernel; on return h_status holds its status words.
int launch_index(gpj_ctx* ctx, bool exact, const gpj::IndexParams& base) {
    const int64_t ntiles = base.ntiles;
    int rc = ensure_tile_state(ctx, ntiles);
    if (rc) return rc;
    GPJ_CUDA(ctx, cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned int), ctx->stream));
    GPJ_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, 2 * sizeof(unsigned long long), ctx->stream));
    gpj::IndexParams p = base;
    p.tile_state = ctx->d_tile_state;
    p.tile_counter = ctx->d_counter;
    p.status = ctx->d_status;
    p.epoch = ctx->epoch;
    const int slot = occupancy_slot(p.num_levels);
    const int occ = exact ? ctx->index_occupancy[slot] : ctx->line_occupancy[slot];
    const int64_t grid = std::min<int64_t>(ntiles, static_cast<int64_t>(ctx->sms) * occ);
    GPJ_CUDA(ctx, exact ? gpj::launch_index_kernel(p, static_cast<int>(grid), ctx->stream)
                        : gpj::launch_line_index_kernel(p, static_cast<int>(grid), ctx->stream));
    ctx->launches++;
    GPJ_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, 2 * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GPJ_OK;
}

// Maps the error word of an index launch to a status code and message.
int status_error(gpj_ctx* ctx, unsigned long long errs) {
    if (!(errs & ~(gpj::kErrDeferred | gpj::kErrOutOverflow))) return GPJ_OK;
    std::string m = "index kernel reported:";
    if (errs & gpj::kErrLookbackTimeout) m += " look-back wait expired;";
    if (errs & gpj::kErrCopyTimeout) m += " TMA copy wait expired;";
    if (errs & (gpj::kErrIrregular | gpj::kErrLongLine)) m += " unexpected line check failure;";
    return fail(ctx, GPJ_EDEVICE, m);
}

// Queries evaluated by the index pass (packed bytecode already on device).
struct FusedQueries {
    int nq = 0;
    int slots = 0;
    const uint8_t* bytecode = nullptr;
    int bytecode_bytes = 0;
    const int32_t* offsets = nullptr;
    int64_t* out = nullptr;
    int64_t out_lines = 0;  // query stride of `out`
};

// Scratch of a standalone index build: the '\n' bitmap, the newline count
// and the newline offset of every tile (pool allocations, freed after the build).
struct TileScratch {
    uint64_t* bits = nullptr;
    int32_t* counts = nullptr;
    int64_t* offsets = nullptr;
};

int alloc_tile_scratch(gpj_ctx* ctx, int64_t n, TileScratch* ts) {
    const int64_t ntiles = (n + gpj::kStandaloneTileBytes - 1) / gpj::kStandaloneTileBytes;
    int rc = device_alloc(ctx, &ts->bits, static_cast<size_t>((n + 63) / 64), "cudaMalloc(newline bitmap)");
    if (!rc) rc = device_alloc(ctx, &ts->counts, static_cast<size_t>(ntiles), "cudaMalloc(tile counts)");
    if (!rc)
        rc = device_alloc(ctx, &ts->offsets, static_cast<size_t>(gpj::newline_offsets_words(ntiles)),
                          "cudaMalloc(tile offsets)");
    return rc;
}

void free_tile_scratch(gpj_ctx* ctx, TileScratch* ts) {
    device_free(ctx, ts->bits);
    device_free(ctx, ts->counts);
    device_free(ctx, ts->offsets);
}

// Parameters of the standalone index kernel over tiles [tile_begin, tile_end).
void set_tile_range(gpj::IndexParams* p, int64_t tile_begin, int64_t tile_end, int64_t avail) {
    p->tile_begin = tile_begin;
    p->tile_end = tile_end;
    p->avail = avail;
}

// Standalone index kernel CTAs per SM (the tuning's choice when it sets one
// below the maximum).
int tile_ctas_per_sm(const gpj_ctx* ctx, int num_levels) {
    const int occ = ctx->tile_occupancy[occupancy_slot(num_levels)];
    const int want = ctx->tuning.index_ctas_per_sm;
    return want > 0 && want < occ ? want : occ;
}

int launch_tiles(gpj_ctx* ctx, const gpj::IndexParams& base) {
    const int occ = tile_ctas_per_sm(ctx, base.num_levels);
    const int64_t grid = std::min<int64_t>(base.tile_end - base.tile_begin, static_cast<int64_t>(ctx->sms) * occ);
    gpj::IndexParams p = base;
    p.tile_counter = tile_claims(ctx);
    GPJ_CUDA(ctx, cudaMemsetAsync(p.tile_counter, 0, sizeof(unsigned int), ctx->stream));
    GPJ_CUDA(ctx, gpj::launch_tile_index_kernel(p, static_cast<int>(grid), ctx->stream));
    ctx->launches++;
    return GPJ_OK;
}

// The newline index from the tiles' bitmap and counts; on return h_status
// holds the status words (line count, error bits).
int finish_tiles(gpj_ctx* ctx, const gpj::IndexParams& p, const TileScratch& ts) {
    const int64_t ntiles = (p.n + gpj::kStandaloneTileBytes - 1) / gpj::kStandaloneTileBytes;
    const int64_t grid = std::min<int64_t>((ntiles + 7) / 8, static_cast<int64_t>(ctx->sms) * 8);
    GPJ_CUDA(ctx, gpj::launch_newline_index(p, ts.offsets, static_cast<int>(grid), ctx->stream));
    ctx->launches += 2;
    GPJ_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, 2 * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GPJ_OK;
}

// Builds the index with the line-parallel kernel (evaluating `fq` in the
// same pass when given), and again with the exact kernel when the input is
// not well-formed NDJSON.  *lines receives the line count; *queries_done
// tells whether every line's query results were written.
// d_colon (optional) receives the ':' bitmap when the standalone kernel
// builds the index; *colon_valid (optional) tells whether it did.
// *exact_only (optional, in and out): the input needs the exact kernel (a
// line kernel flagged it before, so later builds of the same input skip
// straight to the exact kernel).
int run_index(gpj_ctx* ctx, const uint8_t* d_file, int64_t n, int num_levels, uint64_t* d_str,
              uint64_t* d_lvl, int64_t* d_nl, int64_t nl_cap, int64_t* lines, const FusedQueries* fq = nullptr,
              bool* queries_done = nullptr, uint64_t* d_colon = nullptr, bool* colon_valid = nullptr,
              bool* exact_only = nullptr) {
    if (queries_done) *queries_done = false;
    if (colon_valid) *colon_valid = false;
    if (n == 0) {
        if (nl_cap > 0) GPJ_CUDA(ctx, cudaMemsetAsync(d_nl, 0, 8, ctx->stream));
        GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        *lines = 1;
        return GPJ_OK;
    }
    gpj::IndexParams p{};
    p.file = d_file;
    p.n = n;
    p.ntiles = (n + gpj::kIndexTileBytes - 1) / gpj::kIndexTileBytes;
    p.string_index = d_str;
    p.leveled = d_lvl;
    p.level_size = (n + 63) / 64;
    p.num_levels = num_levels;
    p.newlines = d_nl;
    p.newline_cap = nl_cap;
    p.materialize = 1;
    p.tile_begin = 0;
    p.tile_end = p.ntiles;
    p.avail = n;
    gpj::IndexParams fused = p;  // the line-parallel kernel's launch (its own tile size)
    fused.ntiles = (n + gpj::kLineTileBytes - 1) / gpj::kLineTileBytes;
    fused.tile_end = fused.ntiles;
    if (fq && fq->nq > 0) {
        fused.num_queries = fq->nq;
        fused.bytecode = fq->bytecode;
        fused.bytecode_bytes = fq->bytecode_bytes;
        fused.offsets = fq->offsets;
        fused.slots = fq->slots;
        fused.out = fq->out;
        fused.out_lines = fq->out_lines;
    }
    int rc;
    if (exact_only && *exact_only) {
        // known from an earlier build: the line kernels would flag this input
        ctx->exact_fallbacks++;
        rc = launch_index(ctx, true, p);
        if (rc) return rc;
        if ((rc = status_error(ctx, ctx->h_status[1]))) return rc;
        *lines = static_cast<int64_t>(ctx->h_status[0]);
        return GPJ_OK;
    }
    if (fq && fq->nq > 0) {
        rc = launch_index(ctx, false, fused);
        if (rc) return rc;
    } else {
        // index only: the standalone kernel, then the newline index
        TileScratch ts;
        rc = alloc_tile_scratch(ctx, n, &ts);
        if (!rc) {
            const cudaError_t e = cudaMemsetAsync(ctx->d_status, 0, 2 * sizeof(unsigned long long), ctx->stream);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "cudaMemsetAsync(status)");
        }
        if (!rc) {
            fused.ntiles = (n + gpj::kStandaloneTileBytes - 1) / gpj::kStandaloneTileBytes;  // its own tile size
            fused.tile_end = fused.ntiles;
            fused.newline_bits = ts.bits;
            fused.tile_newlines = ts.counts;
            fused.colon = d_colon;
            fused.status = ctx->d_status;
            rc = launch_tiles(ctx, fused);
            if (!rc) rc = finish_tiles(ctx, fused, ts);
        }
        free_tile_scratch(ctx, &ts);
        if (rc) return rc;
    }
    unsigned long long errs = ctx->h_status[1];
    bool exact = false;
    if (errs & (gpj::kErrIrregular | gpj::kErrLongLine)) {
        ctx->exact_fallbacks++;
        exact = true;
        if (exact_only) *exact_only = true;
        rc = launch_index(ctx, true, p);
        if (rc) return rc;
        errs = ctx->h_status[1];
    }
    rc = status_error(ctx, errs);
    if (rc) return rc;
    *lines = static_cast<int64_t>(ctx->h_status[0]);
    if (colon_valid) *colon_valid = d_colon && !exact && !(fq && fq->nq > 0);
    if (queries_done && fq && fq->nq > 0)
        *queries_done = !exact && !(errs & (gpj::kErrDeferred | gpj::kErrOutOverflow)) && *lines <= fq->out_lines;
    return GPJ_OK;
}

int check_ctx(gpj_ctx* ctx) {
    if (!ctx) return GPJ_EINVAL;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    return GPJ_OK;
}

// A file is used with the context that made it (its buffers live in that
// context's pool and are ordered on that context's stream).
int check_file(gpj_ctx* ctx, const gpj_file* f) {
    if (!f || f->ctx != ctx) return fail(ctx, GPJ_EINVAL, "file does not belong to this context");
    return GPJ_OK;
}

int make_file(gpj_ctx* ctx, int64_t n, gpj_file** out) {
    gpj_file* f = new (std::nothrow) gpj_file;
    if (!f) return fail(ctx, GPJ_ENOMEM, "out of host memory");
    f->ctx = ctx;
    f->n = n;
    f->words = (n + 63) / 64;
    *out = f;
    return GPJ_OK;
}

// Packs validated bytecode as [int32 offsets (16-byte padded)][bytes] and
// uploads it unless the previous upload was identical.
int upload_queries(gpj_ctx* ctx, gpj_file* f, int nq, const uint8_t* const* bc, const size_t* len,
                   int slots, int* depth_needed) {
    std::vector<uint8_t> packed;
    const size_t header = ((static_cast<size_t>(nq) * 4 + 15) / 16) * 16;
    packed.resize(header);
    int deepest = 0;
    for (int q = 0; q < nq; q++) {
        if (!bc[q] || len[q] == 0) return fail(ctx, GPJ_EINVAL, "empty bytecode for query " + std::to_string(q));
        int depth = 0, stores = 0;
        std::string why;
        if (!gpj::validate_bytecode(bc[q], len[q], GPJ_MAX_LEVELS, slots, &depth, &stores, &why))
            return fail(ctx, GPJ_EINVAL, "invalid bytecode for query " + std::to_string(q) + ": " + why);
        deepest = std::max(deepest, depth);
        const int32_t off = static_cast<int32_t>(packed.size() - header);
        std::memcpy(packed.data() + 4 * q, &off, 4);
        packed.insert(packed.end(), bc[q], bc[q] + len[q]);
    }
    *depth_needed = deepest;
    f->ir_depth = deepest;
    if (packed == f->ir_host && f->d_ir) return GPJ_OK;
    if (packed.size() > f->d_ir_cap) {
        device_free(ctx, f->d_ir);
        f->d_ir_cap = 0;
        int rc = device_alloc(ctx, &f->d_ir, packed.size() * 2, "cudaMalloc(bytecode)");
        if (rc) return rc;
        f->d_ir_cap = packed.size() * 2;
    }
    GPJ_CUDA(ctx, cudaMemcpyAsync(f->d_ir, packed.data(), packed.size(), cudaMemcpyHostToDevice, ctx->stream));
    GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    f->ir_host.swap(packed);
    return GPJ_OK;
}

// find_value CTAs per SM for queries no deeper than `depth` (the tuning's
// choice when it sets one below the maximum).
int query_occupancy(const gpj_ctx* ctx, int depth) {
    const int occ = ctx->query_occupancy[depth <= 4 ? 0 : (depth <= 8 ? 1 : 2)];
    const int want = ctx->tuning.query_ctas_per_sm;
    return want > 0 && want < occ ? want : occ;
}

// The hand-over of long lines to a warp each, or none (tuning.long_line_bytes < 0).
gpj::LongLines long_lines(const gpj_ctx* ctx) {
    if (ctx->tuning.long_line_bytes < 0 || !ctx->d_long) return gpj::LongLines{nullptr, nullptr, 0, 0};
    return gpj::LongLines{ctx->d_long, ctx->d_long_count, kLongItems, ctx->tuning.long_line_bytes};
}

// find_value over the file's lines, or (d_range given) over lines
// [d_range[0], d_range[1]) of a file whose index is still being built
// (`last`: they include the file's last line).
int launch_query(gpj_ctx* ctx, gpj_file* f, int nq, int slots, int64_t* d_out, int64_t out_lines,
                 const int64_t* d_range = nullptr, bool last = false) {
    cudaStream_t stream = ctx->stream;
    const size_t header = ((static_cast<size_t>(nq) * 4 + 15) / 16) * 16;
    gpj::QueryParams p{};
    p.file = f->d_data;
    p.n = f->n;
    p.newlines = f->d_nl;
    p.num_lines = f->num_lines;
    p.string_index = f->d_str;
    p.leveled = f->d_lvl;
    p.level_size = f->words;
    p.bytecode = f->d_ir + header;
    p.offsets = reinterpret_cast<const int32_t*>(f->d_ir);
    p.num_queries = nq;
    p.slots = slots;
    p.out = d_out;
    p.out_lines = out_lines;
    p.range = d_range;
    p.last = last ? 1 : 0;
    p.newline_cap = f->nl_cap;
    p.colon = f->colon_valid ? f->d_colon : nullptr;
    p.depth = f->ir_depth;
    p.long_lines = long_lines(ctx);
    if (p.long_lines.items)
        GPJ_CUDA(ctx, cudaMemsetAsync(ctx->d_long_count, 0, sizeof(unsigned long long), stream));
    const int64_t want =
        d_range ? INT64_MAX : (gpj::query_items(f->num_lines, nq) + gpj::kQueryThreads - 1) / gpj::kQueryThreads;
    const int64_t grid = std::max<int64_t>(
        1, std::min<int64_t>(want, static_cast<int64_t>(ctx->sms) * query_occupancy(ctx, f->ir_depth)));
    GPJ_CUDA(ctx, gpj::launch_find_value(p, static_cast<int>(grid), ctx->sms * 2, stream));
    ctx->launches += p.long_lines.items ? 2 : 1;
    return GPJ_OK;
}

int check_query_args(gpj_ctx* ctx, int nq, int slots) {
    if (nq < 1 || nq > GPJ_MAX_QUERIES)
        return fail(ctx, GPJ_ELIMIT, "Maximum size of queries is 255 (got " + std::to_string(nq) + ")");
    if (slots < 1) return fail(ctx, GPJ_EINVAL, "result_slots must be >= 1");
    return GPJ_OK;
}

int ensure_index_buffers(gpj_ctx* ctx, gpj_file* f, int num_levels) {
    int rc;
    if (num_levels < 1 || num_levels > GPJ_MAX_LEVELS)
        return fail(ctx, GPJ_ELIMIT, "Invalid number of levels: " + std::to_string(num_levels));
    if (!f->d_str && (rc = device_alloc(ctx, &f->d_str, static_cast<size_t>(f->words), "cudaMalloc(string index)")))
        return rc;
    if (!f->d_colon && (rc = device_alloc(ctx, &f->d_colon, static_cast<size_t>(std::max<int64_t>(f->words, 1)),
                                          "cudaMalloc(colon bitmap)")))
        return rc;
    if (f->lvl_cap < num_levels) {
        device_free(ctx, f->d_lvl);
        f->lvl_cap = 0;
        rc = device_alloc(ctx, &f->d_lvl, static_cast<size_t>(f->words) * num_levels, "cudaMalloc(leveled bitmaps)");
        if (rc) return rc;
        f->lvl_cap = num_levels;
    }
    if (!f->d_nl) {
        f->nl_cap = std::min<int64_t>(f->n + 1, f->n / 256 + 1024);
        rc = device_alloc(ctx, &f->d_nl, static_cast<size_t>(f->nl_cap), "cudaMalloc(newline index)");
        if (rc) return rc;
    }
    return GPJ_OK;
}

// The index pass of a file (and the queries in `fq`, when given, in the same
// pass).  Grows the newline index and repeats the pass when the file has
// more lines than the first estimate.
int index_pass(gpj_ctx* ctx, gpj_file* f, int num_levels, const FusedQueries* fq, bool* queries_done) {
    int rc = ensure_index_buffers(ctx, f, num_levels);
    if (rc) return rc;
    f->indexed = false;
    f->colon_valid = false;
    const double t0 = now_ms();
    GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    int64_t lines = 0;
    rc = run_index(ctx, f->d_data, f->n, num_levels, f->d_str, f->d_lvl, f->d_nl, f->nl_cap, &lines, fq,
                   queries_done, f->d_colon, &f->colon_valid, &f->exact_only);
    if (rc) return rc;
    if (lines > f->nl_cap) {  // more lines than the first guess: size exactly and rebuild
        device_free(ctx, f->d_nl);
        f->nl_cap = lines;
        rc = device_alloc(ctx, &f->d_nl, static_cast<size_t>(lines), "cudaMalloc(newline index)");
        if (rc) return rc;
        rc = run_index(ctx, f->d_data, f->n, num_levels, f->d_str, f->d_lvl, f->d_nl, f->nl_cap, &lines, fq,
                       queries_done, f->d_colon, &f->colon_valid, &f->exact_only);
        if (rc) return rc;
    }
    rc = end_phase(ctx, fq && fq->nq ? "index_and_query" : "build_index", t0);
    if (rc) return rc;
    f->num_lines = lines;
    f->num_levels = num_levels;
    f->indexed = true;
    return GPJ_OK;
}

// Tiles copied per step of load_and_index: 2048 standalone-kernel tiles
// (60 MiB), a whole number of the newline scan's 1024-tile blocks.
constexpr int64_t kLoadTiles = 2048;

// Queries load_and_index evaluates on each chunk's lines as soon as their
// index is complete (bytecode uploaded; results strided by out_lines).
struct ChunkQueries {
    int nq = 0;
    int slots = 0;
    int64_t* d_out = nullptr;
    int64_t out_lines = 0;
};

// Copies n host bytes into f->d_owned in chunks on the copy stream and
// indexes chunk k with the line-parallel kernel as soon as chunk k + 1 has
// landed (a line starting in chunk k ends in chunk k + 1 unless it is longer
// than a chunk), so the copy and the index build overlap.  With `cq`, the
// newline index of chunk k follows at once, and then find_value on the
// lines it completes, so the queries overlap the copy too (*queries_done
// tells whether they all ran that way).  Inputs the line kernel cannot
// index this way (not NDJSON, or a line longer than a chunk) are indexed
// again from the complete copy by run_index.
//
// host == nullptr: the input is already in f->d_data; chunks of
// `chunk_tiles` tiles are indexed and queried in turn (index kernel, newline
// index, find_value on the lines the chunk completes), so find_value reads a
// chunk's index while it is still in L2.
int load_and_index(gpj_ctx* ctx, gpj_file* f, const uint8_t* host, int num_levels, const ChunkQueries* cq = nullptr,
                   bool* queries_done = nullptr, int64_t chunk_tiles = kLoadTiles) {
    const int64_t n = f->n;
    const bool resident = host == nullptr;
    if (queries_done) *queries_done = false;
    int rc = ensure_index_buffers(ctx, f, num_levels);
    if (rc) return rc;
    f->indexed = false;
    f->colon_valid = false;
    const double t0 = now_ms();
    GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    const int64_t chunk_bytes = gpj::kStandaloneTileBytes * chunk_tiles;
    const int64_t nchunks = (n + chunk_bytes - 1) / chunk_bytes;
    int64_t lines = 0;
    if (nchunks <= 1) {
        if (n > 0 && !resident)
            GPJ_CUDA(ctx, cudaMemcpyAsync(f->d_owned, host, static_cast<size_t>(n), cudaMemcpyHostToDevice,
                                          ctx->stream));
        rc = run_index(ctx, f->d_data, n, num_levels, f->d_str, f->d_lvl, f->d_nl, f->nl_cap, &lines, nullptr,
                           nullptr, f->d_colon, &f->colon_valid, &f->exact_only);
        if (rc) return rc;
    } else {
        while (!resident && static_cast<int64_t>(ctx->chunk_events.size()) < nchunks) {
            cudaEvent_t e = nullptr;
            GPJ_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            ctx->chunk_events.push_back(e);
        }
        gpj::IndexParams p{};
        p.file = f->d_data;
        p.n = n;
        p.ntiles = (n + gpj::kStandaloneTileBytes - 1) / gpj::kStandaloneTileBytes;
        p.string_index = f->d_str;
        p.leveled = f->d_lvl;
        p.level_size = f->words;
        p.num_levels = num_levels;
        p.newlines = f->d_nl;
        p.newline_cap = f->nl_cap;
        p.materialize = 1;
        p.colon = f->d_colon;
        f->colon_valid = true;  // the chunks' queries read it as their tiles write it
        TileScratch ts;
        rc = alloc_tile_scratch(ctx, n, &ts);
        int64_t* d_lines = nullptr;  // [k + 1]: lines complete after chunk k
        if (!rc && cq) rc = device_alloc(ctx, &d_lines, static_cast<size_t>(nchunks + 1), "cudaMalloc(chunk lines)");
        if (!rc) {
            cudaError_t e = cq ? cudaMemsetAsync(d_lines, 0, sizeof(int64_t), ctx->stream) : cudaSuccess;
            if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_status, 0, 2 * sizeof(unsigned long long), ctx->stream);
            // the copies start once the buffers exist (pool allocations are ordered on ctx->stream)
            if (e == cudaSuccess && !resident) e = cudaEventRecord(ctx->ev_ready, ctx->stream);
            if (e == cudaSuccess && !resident) e = cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_ready, 0);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "chunked index setup");
        }
        if (rc) {
            free_tile_scratch(ctx, &ts);
            device_free(ctx, d_lines);
            f->colon_valid = false;
            return rc;
        }
        p.status = ctx->d_status;
        p.newline_bits = ts.bits;
        p.tile_newlines = ts.counts;
        auto launch_chunk = [&](int64_t k) -> int {
            const int64_t t0 = k * chunk_tiles, t1 = std::min(p.ntiles, (k + 1) * chunk_tiles);
            set_tile_range(&p, t0, t1, resident ? n : std::min(n, (k + 2) * chunk_bytes));
            if (!resident)
                GPJ_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->chunk_events[std::min(k + 1, nchunks - 1)], 0));
            int r = launch_tiles(ctx, p);
            if (r || !cq) return r;
            // the chunk's newline index, then the queries on the lines it completes
            const int64_t grid = std::min<int64_t>((t1 - t0 + 7) / 8, static_cast<int64_t>(ctx->sms) * 8);
            GPJ_CUDA(ctx, gpj::launch_newline_index_range(p, ts.offsets, t0, t1, d_lines + k + 1, static_cast<int>(grid),
                                                          ctx->stream));
            ctx->launches += 2;
            return launch_query(ctx, f, cq->nq, cq->slots, cq->d_out, cq->out_lines, d_lines + k, k == nchunks - 1);
        };
        for (int64_t k = 0; k < nchunks && !rc; k++) {
            if (resident) {
                rc = launch_chunk(k);
                continue;
            }
            const int64_t pos = k * chunk_bytes;
            const size_t len = static_cast<size_t>(std::min(chunk_bytes, n - pos));
            cudaError_t e = cudaMemcpyAsync(f->d_owned + pos, host + pos, len, cudaMemcpyHostToDevice, ctx->copy_stream);
            if (e == cudaSuccess) e = cudaEventRecord(ctx->chunk_events[k], ctx->copy_stream);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "cudaMemcpyAsync(file chunk)");
            if (!rc && k >= 1) rc = launch_chunk(k - 1);
        }
        if (!rc && !resident) rc = launch_chunk(nchunks - 1);
        if (!rc) {
            if (cq) {  // the newline index is complete: read the status words
                cudaError_t e = cudaMemcpyAsync(ctx->h_status, ctx->d_status, 2 * sizeof(unsigned long long),
                                                cudaMemcpyDeviceToHost, ctx->stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
                if (e != cudaSuccess) rc = cuda_fail(ctx, e, "chunked index status");
            } else {
                rc = finish_tiles(ctx, p, ts);
            }
        }
        free_tile_scratch(ctx, &ts);
        device_free(ctx, d_lines);
        if (rc) {
            f->colon_valid = false;
            if (!resident) cudaStreamSynchronize(ctx->copy_stream);
            return rc;
        }
        const unsigned long long errs = ctx->h_status[1];
        lines = static_cast<int64_t>(ctx->h_status[0]);
        if (errs & (gpj::kErrIrregular | gpj::kErrLongLine)) {
            // the whole input is on the device now: index it in one launch (exact fallback inside)
            rc = run_index(ctx, f->d_data, n, num_levels, f->d_str, f->d_lvl, f->d_nl, f->nl_cap, &lines, nullptr,
                           nullptr, f->d_colon, &f->colon_valid, &f->exact_only);
            if (rc) return rc;
        } else if ((rc = status_error(ctx, errs))) {
            f->colon_valid = false;
            return rc;
        } else if (cq && lines <= f->nl_cap && lines <= cq->out_lines && queries_done) {
            *queries_done = true;
        }
    }
    if (lines > f->nl_cap) {  // more lines than the first guess: size exactly and rebuild
        device_free(ctx, f->d_nl);
        f->nl_cap = lines;
        rc = device_alloc(ctx, &f->d_nl, static_cast<size_t>(lines), "cudaMalloc(newline index)");
        if (rc) return rc;
        rc = run_index(ctx, f->d_data, n, num_levels, f->d_str, f->d_lvl, f->d_nl, f->nl_cap, &lines, nullptr,
                           nullptr, f->d_colon, &f->colon_valid, &f->exact_only);
        if (rc) return rc;
    }
    rc = end_phase(ctx, resident ? "index_and_query" : "load_and_index", t0);
    if (rc) return rc;
    f->num_lines = lines;
    f->num_levels = num_levels;
    f->indexed = true;
    return GPJ_OK;
}

// Index + queries in one pass when possible, into d_out with query stride
// out_lines (>= the line count, else GPJ_ELIMIT with *lines_needed set).
int index_and_query(gpj_ctx* ctx, gpj_file* f, int num_levels, int nq, const uint8_t* const* bc,
                    const size_t* len, int slots, int64_t* d_out, int64_t out_lines, int64_t* lines_needed) {
    int rc = check_query_args(ctx, nq, slots);
    if (rc) return rc;
    int depth = 0;
    rc = upload_queries(ctx, f, nq, bc, len, slots, &depth);
    if (rc) return rc;
    if (depth > num_levels)
        return fail(ctx, GPJ_ELIMIT, "queries need " + std::to_string(depth) + " levels, the index is built with " +
                                         std::to_string(num_levels));
    const int64_t chunk_tiles = ctx->tuning.chunk_tiles;
    if (!ctx->fuse_queries && chunk_tiles > 0 && !f->exact_only &&
        f->n > gpj::kStandaloneTileBytes * chunk_tiles) {
        // chunk by chunk: index kernel, newline index, find_value on the
        // lines the chunk completes
        ChunkQueries cq;
        cq.nq = nq;
        cq.slots = slots;
        cq.d_out = d_out;
        cq.out_lines = out_lines;
        bool done = false;
        rc = load_and_index(ctx, f, nullptr, num_levels, &cq, &done, chunk_tiles);
        if (rc) return rc;
        if (lines_needed) *lines_needed = f->num_lines;
        if (f->num_lines > out_lines)
            return fail(ctx, GPJ_ELIMIT, "result buffer holds " + std::to_string(out_lines) +
                                             " lines, the file has " + std::to_string(f->num_lines));
        if (done) return GPJ_OK;
        const double t1 = now_ms();
        GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
        rc = launch_query(ctx, f, nq, slots, d_out, out_lines);
        if (rc) return rc;
        return end_phase(ctx, "find_value", t1);
    }
    if (!ctx->fuse_queries) {
        // index kernel, then one find_value launch for all queries
        rc = index_pass(ctx, f, num_levels, nullptr, nullptr);
        if (rc) return rc;
        if (lines_needed) *lines_needed = f->num_lines;
        if (f->num_lines > out_lines)
            return fail(ctx, GPJ_ELIMIT, "result buffer holds " + std::to_string(out_lines) +
                                             " lines, the file has " + std::to_string(f->num_lines));
        const double t1 = now_ms();
        GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
        rc = launch_query(ctx, f, nq, slots, d_out, out_lines);
        if (rc) return rc;
        return end_phase(ctx, "find_value", t1);
    }
    FusedQueries fq;
    fq.nq = nq;
    fq.slots = slots;
    const size_t header = ((static_cast<size_t>(nq) * 4 + 15) / 16) * 16;
    fq.offsets = reinterpret_cast<const int32_t*>(f->d_ir);
    fq.bytecode = f->d_ir + header;
    fq.bytecode_bytes = static_cast<int>(f->ir_host.size() - header);
    fq.out = d_out;
    fq.out_lines = out_lines;
    bool done = false;
    rc = index_pass(ctx, f, num_levels, &fq, &done);
    if (rc) return rc;
    if (lines_needed) *lines_needed = f->num_lines;
    if (f->num_lines > out_lines)
        return fail(ctx, GPJ_ELIMIT, "result buffer holds " + std::to_string(out_lines) + " lines, the file has " +
                                         std::to_string(f->num_lines));
    if (!done) {
        // lines the fused pass could not evaluate (or an input that needed the
        // exact kernel): evaluate every line from the materialised index
        const double t1 = now_ms();
        GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
        rc = launch_query(ctx, f, nq, slots, d_out, out_lines);
        if (rc) return rc;
        rc = end_phase(ctx, "find_value", t1);
        if (rc) return rc;
    }
    return GPJ_OK;
}

int query_common(gpj_ctx* ctx, gpj_file* f, int nq, const uint8_t* const* bc, const size_t* len,
                 int slots, int64_t* d_out, int64_t out_count, bool to_host, int64_t* host_out) {
    int rc = check_query_args(ctx, nq, slots);
    if (rc) return rc;
    if (!f->indexed) return fail(ctx, GPJ_ESTATE, "file is not indexed (call gpj_index_build)");
    const int64_t need = static_cast<int64_t>(nq) * f->num_lines * slots * 2;
    if (out_count < need)
        return fail(ctx, GPJ_EINVAL, "output holds " + std::to_string(out_count) + " elements, " +
                                         std::to_string(need) + " needed");
    int depth = 0;
    rc = upload_queries(ctx, f, nq, bc, len, slots, &depth);
    if (rc) return rc;
    if (depth > f->num_levels)
        return fail(ctx, GPJ_ESTATE, "queries need " + std::to_string(depth) + " levels, index has " +
                                         std::to_string(f->num_levels));
    const double t0 = now_ms();
    GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    rc = launch_query(ctx, f, nq, slots, d_out, f->num_lines);
    if (rc) return rc;
    if (!to_host) return GPJ_OK;
    rc = end_phase(ctx, "find_value", t0);
    if (rc) return rc;
    const double t1 = now_ms();
    GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    GPJ_CUDA(ctx, cudaMemcpyAsync(host_out, d_out, need * 8, cudaMemcpyDeviceToHost, ctx->stream));
    return end_phase(ctx, "copy_results", t1);
}

int ensure_out(gpj_ctx* ctx, gpj_file* f, size_t elems) {
    if (elems <= f->d_out_cap) return GPJ_OK;
    device_free(ctx, f->d_out);
    f->d_out_cap = 0;
    int rc = device_alloc(ctx, &f->d_out, elems, "cudaMalloc(results)");
    if (rc) return rc;
    f->d_out_cap = elems;
    return GPJ_OK;
}

// Value extraction over result pairs of file f (values.cu): kinds and
// offsets, then (d_bytes_out given) a device buffer of exactly the total is
// allocated into *d_bytes_out, else the values go into d_bytes (cap bytes;
// null when cap is 0).  *total receives the byte total; synchronous.
int gather_values(gpj_ctx* ctx, gpj_file* f, const int64_t* d_pairs, int64_t npairs, int64_t per_query,
                  int64_t stride, uint8_t* d_kinds, int64_t* d_offsets, uint8_t* d_bytes, int64_t cap,
                  uint8_t** d_bytes_out, int64_t* total) {
    int64_t* scratch = nullptr;  // [block sums..., total]
    const int64_t blocks = gpj::value_scan_blocks(npairs);
    int rc = device_alloc(ctx, &scratch, static_cast<size_t>(blocks + 1), "cudaMalloc(value scan)");
    if (rc) return rc;
    int64_t* d_total = scratch + blocks;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((npairs + 255) / 256, static_cast<int64_t>(ctx->sms) * 8));
    auto run = [&]() -> int {
        GPJ_CUDA(ctx, gpj::launch_value_sizes(d_pairs, npairs, std::max<int64_t>(per_query, 1), stride, f->n, d_kinds,
                                              d_offsets, scratch, d_total, ctx->stream));
        ctx->launches += npairs > 0 ? 2 : 1;
        if (d_bytes_out) {
            GPJ_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, d_total, 8, cudaMemcpyDeviceToHost, ctx->stream));
            GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            *total = static_cast<int64_t>(ctx->h_status[0]);
            int r = device_alloc(ctx, d_bytes_out, static_cast<size_t>(std::max<int64_t>(*total, 1)),
                                 "cudaMalloc(values)");
            if (r) return r;
            d_bytes = *d_bytes_out;
            cap = *total;
        }
        GPJ_CUDA(ctx, gpj::launch_value_copy(f->d_data, d_pairs, npairs, std::max<int64_t>(per_query, 1), stride,
                                             d_kinds, d_offsets, scratch, d_total, d_bytes, cap, static_cast<int>(grid),
                                             ctx->stream));
        ctx->launches++;
        GPJ_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, d_total, 8, cudaMemcpyDeviceToHost, ctx->stream));
        GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        *total = static_cast<int64_t>(ctx->h_status[0]);
        return GPJ_OK;
    };
    rc = run();
    device_free(ctx, scratch);
    return rc;
}


}  // namespace

extern "C" {

const char* gpj_version(void) { return "gpjson_b200 0.1 sm_100a"; }

int gpj_create(int device, gpj_ctx** out) {
    if (!out) return GPJ_EINVAL;
    *out = nullptr;
    gpj_ctx* ctx = new (std::nothrow) gpj_ctx;
    if (!ctx) return GPJ_ENOMEM;
    auto bail = [&](cudaError_t e, const char* what) {
        cuda_fail(ctx, e, what);
        g_create_error = ctx->err;
        gpj_destroy(ctx);
        return e == cudaErrorMemoryAllocation ? GPJ_ENOMEM : GPJ_ECUDA;
    };
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bail(e, "cudaSetDevice");
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return bail(e, "cudaGetDeviceProperties");
    if (prop.major != 10) {
        g_create_error = std::string("device ") + prop.name + " is not sm_100 (this library is built for sm_100a only)";
        gpj_destroy(ctx);
        return GPJ_ECUDA;
    }
    ctx->sms = prop.multiProcessorCount;
    if ((e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(e, "cudaStreamCreate");
    ctx->stream = ctx->own_stream;
    if ((e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(e, "cudaStreamCreate(copy)");
    if ((e = cudaEventCreateWithFlags(&ctx->ev_ready, cudaEventDisableTiming)) != cudaSuccess)
        return bail(e, "cudaEventCreate");
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        if ((e = cudaMemPoolCreate(&ctx->pool, &props)) != cudaSuccess) return bail(e, "cudaMemPoolCreate");
        uint64_t keep = UINT64_MAX;  // freed blocks stay in the pool until gpj_destroy
        if ((e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess)
            return bail(e, "cudaMemPoolSetAttribute");
    }
    if ((e = cudaMalloc(&ctx->d_counter, 16)) != cudaSuccess) return bail(e, "cudaMalloc(counter)");
    if ((e = cudaMalloc(&ctx->d_long, sizeof(gpj::LongItem) * kLongItems)) != cudaSuccess)
        return bail(e, "cudaMalloc(long lines)");
    if ((e = cudaMalloc(&ctx->d_long_count, sizeof(unsigned long long))) != cudaSuccess)
        return bail(e, "cudaMalloc(long line count)");
    ctx->tuning = default_tuning();
    if ((e = cudaMalloc(&ctx->d_status, 16)) != cudaSuccess) return bail(e, "cudaMalloc(status)");
    if ((e = cudaMallocHost(&ctx->h_status, 16)) != cudaSuccess) return bail(e, "cudaMallocHost(status)");
    if ((e = cudaEventCreate(&ctx->ev0)) != cudaSuccess) return bail(e, "cudaEventCreate");
    if ((e = cudaEventCreate(&ctx->ev1)) != cudaSuccess) return bail(e, "cudaEventCreate");
    const int levels[3] = {4, 8, 16};
    for (int i = 0; i < 3; i++) {
        ctx->index_occupancy[i] = gpj::index_kernel_max_ctas_per_sm(levels[i]);
        if (ctx->index_occupancy[i] < 1) return bail(cudaGetLastError(), "index kernel occupancy");
        ctx->line_occupancy[i] = gpj::line_index_max_ctas_per_sm(levels[i]);
        ctx->tile_occupancy[i] = gpj::tile_index_max_ctas_per_sm(levels[i]);
        if (ctx->tile_occupancy[i] < 1) return bail(cudaGetLastError(), "tile index kernel occupancy");
        if (ctx->line_occupancy[i] < 1) return bail(cudaGetLastError(), "line index kernel occupancy");
    }
    for (int v = 0; v < 3; v++) {
        ctx->query_occupancy[v] = gpj::find_value_max_ctas_per_sm(v == 0 ? 4 : (v == 1 ? 8 : GPJ_MAX_LEVELS));
        if (ctx->query_occupancy[v] < 1) return bail(cudaGetLastError(), "find_value occupancy");
    }
    *out = ctx;
    return GPJ_OK;
}

void gpj_destroy(gpj_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream) {
        ctx->stream = ctx->own_stream;
        device_free(ctx, ctx->d_tile_state);
        cudaStreamSynchronize(ctx->own_stream);
    }
    if (ctx->d_counter) cudaFree(ctx->d_counter);
    if (ctx->d_long) cudaFree(ctx->d_long);
    if (ctx->d_long_count) cudaFree(ctx->d_long_count);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    for (cudaEvent_t e : ctx->chunk_events) cudaEventDestroy(e);
    if (ctx->ev_ready) cudaEventDestroy(ctx->ev_ready);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

const char* gpj_last_error(const gpj_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int gpj_set_tuning(gpj_ctx* ctx, const gpj_tuning* tuning) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!tuning) return fail(ctx, GPJ_EINVAL, "tuning is null");
    if (tuning->query_ctas_per_sm < 0 || tuning->index_ctas_per_sm < 0)
        return fail(ctx, GPJ_EINVAL, "CTAs per SM must be >= 0");
    if (tuning->chunk_tiles < 0 || tuning->chunk_tiles % 1024 != 0)
        return fail(ctx, GPJ_EINVAL, "chunk_tiles must be a multiple of 1024 (0 = whole-file passes)");
    ctx->tuning = *tuning;
    if (ctx->tuning.long_line_bytes == 0) ctx->tuning.long_line_bytes = default_tuning().long_line_bytes;
    return GPJ_OK;
}

int gpj_get_tuning(const gpj_ctx* ctx, gpj_tuning* out) {
    if (!ctx || !out) return GPJ_EINVAL;
    *out = ctx->tuning;
    return GPJ_OK;
}

int gpj_set_query_fusion(gpj_ctx* ctx, int enabled) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    ctx->fuse_queries = enabled != 0;
    return GPJ_OK;
}

static_assert(GPJ_PATH_INDEX_UNIONS == gpj::kPathIndexUnions, "extension flags of the ABI and the compiler");

int gpj_set_path_extensions(gpj_ctx* ctx, unsigned extensions) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (extensions & ~GPJ_PATH_INDEX_UNIONS) return fail(ctx, GPJ_EINVAL, "unknown JSONPath extension flags");
    ctx->path_extensions = extensions;
    return GPJ_OK;
}

int gpj_set_stream(gpj_ctx* ctx, void* stream) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    // work (and pool frees) queued on the old stream finish first
    GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return GPJ_OK;
}

int gpj_compile(const char* path, uint8_t* out, size_t cap, size_t* len, int* max_depth,
                int* num_results, char* err, size_t err_cap) {
    return gpj_compile_ex(path, 0, out, cap, len, max_depth, num_results, err, err_cap);
}

int gpj_compile_ex(const char* path, unsigned extensions, uint8_t* out, size_t cap, size_t* len, int* max_depth,
                   int* num_results, char* err, size_t err_cap) {
    auto set_err = [&](const std::string& m) {
        if (err && err_cap > 0) {
            std::strncpy(err, m.c_str(), err_cap - 1);
            err[err_cap - 1] = '\0';
        }
    };
    if (!path || !len || !max_depth || !num_results) {
        set_err("null argument");
        return GPJ_EINVAL;
    }
    try {
        if (extensions & ~GPJ_PATH_INDEX_UNIONS) {
            set_err("unknown JSONPath extension flags");
            return GPJ_EINVAL;
        }
        gpj::CompiledPath r = gpj::compile_path(path, extensions);
        *len = r.bytecode.size();
        *max_depth = r.max_depth;
        *num_results = r.num_results;
        if (r.bytecode.size() > cap || (!out && cap > 0)) {
            set_err("bytecode needs " + std::to_string(r.bytecode.size()) + " bytes");
            return GPJ_ELIMIT;
        }
        if (out) std::memcpy(out, r.bytecode.data(), r.bytecode.size());
        set_err("");
        return GPJ_OK;
    } catch (const gpj::PathError& e) {
        set_err(e.what());
        return e.unsupported ? GPJ_EUNSUPPORTED : GPJ_EPARSE;
    } catch (const std::exception& e) {
        set_err(e.what());
        return GPJ_EPARSE;
    }
}

int gpj_file_from_device(gpj_ctx* ctx, const void* d_data, int64_t n, gpj_file** out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || n < 0 || (n > 0 && !d_data)) return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (reinterpret_cast<uintptr_t>(d_data) % 16 != 0)
        return fail(ctx, GPJ_EINVAL, "device input must be 16-byte aligned");
    rc = make_file(ctx, n, out);
    if (rc) return rc;
    (*out)->d_data = static_cast<const uint8_t*>(d_data);
    return GPJ_OK;
}

int gpj_file_from_host(gpj_ctx* ctx, const void* data, int64_t n, gpj_file** out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || n < 0 || (n > 0 && !data)) return fail(ctx, GPJ_EINVAL, "bad arguments");
    gpj_file* f = nullptr;
    rc = make_file(ctx, n, &f);
    if (rc) return rc;
    rc = device_alloc(ctx, &f->d_owned, static_cast<size_t>(n), "cudaMalloc(file)");
    if (rc) {
        delete f;
        return rc;
    }
    f->d_data = f->d_owned;
    const double t0 = now_ms();
    cudaEventRecord(ctx->ev0, ctx->stream);
    cudaError_t e = cudaMemcpyAsync(f->d_owned, data, static_cast<size_t>(n), cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        gpj_file_release(f);
        return cuda_fail(ctx, e, "cudaMemcpyAsync(file)");
    }
    rc = end_phase(ctx, "copy_file", t0);
    if (rc) {
        gpj_file_release(f);
        return rc;
    }
    *out = f;
    return GPJ_OK;
}

int gpj_file_from_host_indexed(gpj_ctx* ctx, const void* data, int64_t n, int num_levels, gpj_file** out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || n < 0 || (n > 0 && !data)) return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (num_levels < 1 || num_levels > GPJ_MAX_LEVELS)
        return fail(ctx, GPJ_ELIMIT, "Invalid number of levels: " + std::to_string(num_levels));
    gpj_file* f = nullptr;
    rc = make_file(ctx, n, &f);
    if (rc) return rc;
    rc = device_alloc(ctx, &f->d_owned, static_cast<size_t>(n), "cudaMalloc(file)");
    if (rc) {
        delete f;
        return rc;
    }
    f->d_data = f->d_owned;
    rc = load_and_index(ctx, f, static_cast<const uint8_t*>(data), num_levels);
    if (rc) {
        gpj_file_release(f);
        return rc;
    }
    *out = f;
    return GPJ_OK;
}

int gpj_file_from_host_query(gpj_ctx* ctx, const void* data, int64_t n, int num_levels, int nq,
                             const uint8_t* const* bytecode, const size_t* bytecode_len, int result_slots,
                             int64_t* host_out, int64_t out_count, int64_t* num_lines, gpj_file** out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || !num_lines || !bytecode || !bytecode_len || n < 0 || (n > 0 && !data) || out_count < 0 ||
        (out_count > 0 && !host_out))
        return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (num_levels < 1 || num_levels > GPJ_MAX_LEVELS)
        return fail(ctx, GPJ_ELIMIT, "Invalid number of levels: " + std::to_string(num_levels));
    rc = check_query_args(ctx, nq, result_slots);
    if (rc) return rc;
    gpj_file* f = nullptr;
    rc = make_file(ctx, n, &f);
    if (rc) return rc;
    rc = device_alloc(ctx, &f->d_owned, static_cast<size_t>(n), "cudaMalloc(file)");
    if (rc) {
        delete f;
        return rc;
    }
    f->d_data = f->d_owned;
    auto done = [&](int r) {
        if (r) {
            gpj_file_release(f);
            return r;
        }
        *out = f;
        return GPJ_OK;
    };
    int depth = 0;
    rc = upload_queries(ctx, f, nq, bytecode, bytecode_len, result_slots, &depth);
    if (!rc && depth > num_levels)
        rc = fail(ctx, GPJ_ELIMIT, "queries need " + std::to_string(depth) + " levels, the index is built with " +
                                       std::to_string(num_levels));
    if (!rc) rc = ensure_index_buffers(ctx, f, num_levels);
    // results strided by the newline index's line capacity until the count is known
    int64_t stride = f->nl_cap;
    if (!rc) rc = ensure_out(ctx, f, static_cast<size_t>(nq) * stride * result_slots * 2);
    if (rc) return done(rc);
    const double t0 = now_ms();
    ChunkQueries cq;
    cq.nq = nq;
    cq.slots = result_slots;
    cq.d_out = f->d_out;
    cq.out_lines = stride;
    bool queried = false;
    rc = load_and_index(ctx, f, static_cast<const uint8_t*>(data), num_levels, &cq, &queried);
    if (rc) return done(rc);
    if (!queried) {
        // the input was indexed again from the complete copy: query it whole
        stride = f->num_lines;
        rc = ensure_out(ctx, f, static_cast<size_t>(nq) * stride * result_slots * 2);
        if (!rc) rc = launch_query(ctx, f, nq, result_slots, f->d_out, stride);
        if (rc) return done(rc);
    }
    *num_lines = f->num_lines;
    const size_t per_query = static_cast<size_t>(f->num_lines) * result_slots * 2;
    if (out_count < static_cast<int64_t>(per_query * nq)) {
        *out = f;  // indexed and kept: gpj_query gives the results
        return fail(ctx, GPJ_ELIMIT, "output holds " + std::to_string(out_count) + " elements, " +
                                         std::to_string(per_query * nq) + " needed (the file is indexed)");
    }
    for (int q = 0; q < nq && !rc; q++) {
        cudaError_t e = cudaMemcpyAsync(host_out + q * per_query, f->d_out + static_cast<size_t>(q) * stride * result_slots * 2,
                                        per_query * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "cudaMemcpyAsync(results)");
    }
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "cudaStreamSynchronize(results)");
    }
    if (!rc) rc = end_phase(ctx, "load_index_query", t0);
    return done(rc);
}

int gpj_file_open(gpj_ctx* ctx, const char* filename, gpj_file** out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!filename || !out) return fail(ctx, GPJ_EINVAL, "bad arguments");
    const int fd = ::open(filename, O_RDONLY | O_CLOEXEC);
    if (fd < 0) return fail(ctx, GPJ_EIO, std::string("Failed to open file ") + filename);
    struct stat st;
    if (::fstat(fd, &st) != 0 || !S_ISREG(st.st_mode) || st.st_size < 0) {
        ::close(fd);
        return fail(ctx, GPJ_EIO, std::string("Failed to get size of file ") + filename);
    }
    const int64_t n = static_cast<int64_t>(st.st_size);
    gpj_file* f = nullptr;
    rc = make_file(ctx, n, &f);
    if (rc) {
        ::close(fd);
        return rc;
    }
    rc = device_alloc(ctx, &f->d_owned, static_cast<size_t>(n), "cudaMalloc(file)");
    if (rc) {
        ::close(fd);
        delete f;
        return rc;
    }
    f->d_data = f->d_owned;
    // Two pinned halves: the read of one chunk overlaps the copy of the other.
    const size_t chunk = 32u << 20;
    if (!ctx->h_stage) {
        cudaError_t e = cudaMallocHost(&ctx->h_stage, 2 * chunk);
        if (e != cudaSuccess) {
            ::close(fd);
            gpj_file_release(f);
            return cuda_fail(ctx, e, "cudaMallocHost(staging)");
        }
        ctx->stage_bytes = 2 * chunk;
    }
    // one reader thread per 2 MiB of a chunk, at most one per host thread (and 16)
    const int threads = static_cast<int>(std::min<int64_t>(
        std::min<int64_t>(16, std::max(1u, std::thread::hardware_concurrency())), std::max<int64_t>(1, n >> 21)));
    const double t0 = now_ms();
    cudaEventRecord(ctx->ev0, ctx->stream);
    // done[h]: the copy out of staging half h has finished (a half is
    // refilled only after that)
    cudaEvent_t done[2] = {nullptr, nullptr};
    cudaError_t ce = cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming);
    rc = ce == cudaSuccess ? GPJ_OK : cuda_fail(ctx, ce, "cudaEventCreate(file chunks)");
    if (!rc) {
        gpj::SliceReader reader(fd, threads);
        int64_t pos = 0;
        int half = 0;
        while (pos < n) {
            const size_t want = static_cast<size_t>(std::min<int64_t>(static_cast<int64_t>(chunk), n - pos));
            uint8_t* stage = ctx->h_stage + half * chunk;
            cudaError_t e = cudaEventSynchronize(done[half]);
            if (e != cudaSuccess) {
                rc = cuda_fail(ctx, e, "cudaEventSynchronize(file chunk)");
                break;
            }
            if (!reader.read(stage, pos, want)) {
                rc = fail(ctx, GPJ_EIO, std::string("Size of file has changed while reading ") + filename);
                break;
            }
            e = cudaMemcpyAsync(f->d_owned + pos, stage, want, cudaMemcpyHostToDevice, ctx->stream);
            if (e == cudaSuccess) e = cudaEventRecord(done[half], ctx->stream);
            if (e != cudaSuccess) {
                rc = cuda_fail(ctx, e, "cudaMemcpyAsync(file)");
                break;
            }
            pos += static_cast<int64_t>(want);
            half ^= 1;
        }
    }
    ::close(fd);
    if (rc == GPJ_OK) rc = end_phase(ctx, "read_file", t0);
    else cudaStreamSynchronize(ctx->stream);  // no copy still reads the staging
    if (done[0]) cudaEventDestroy(done[0]);
    if (done[1]) cudaEventDestroy(done[1]);
    if (rc) {
        gpj_file_release(f);
        return rc;
    }
    *out = f;
    return GPJ_OK;
}

void gpj_file_release(gpj_file* f) {
    if (!f) return;
    if (f->ctx) {
        cudaSetDevice(f->ctx->device);
        cudaStreamSynchronize(f->ctx->stream);
    }
    if (f->ctx) {
        gpj_ctx* ctx = f->ctx;
        device_free(ctx, f->d_owned);
        device_free(ctx, f->d_str);
        device_free(ctx, f->d_colon);
        device_free(ctx, f->d_lvl);
        device_free(ctx, f->d_nl);
        device_free(ctx, f->d_ir);
        device_free(ctx, f->d_out);
    }
    delete f;
}

int64_t gpj_file_size(const gpj_file* f) { return f ? f->n : -1; }

int gpj_index_build(gpj_ctx* ctx, gpj_file* f, int num_levels) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!f || f->ctx != ctx) return fail(ctx, GPJ_EINVAL, "file does not belong to this context");
    return index_pass(ctx, f, num_levels, nullptr, nullptr);
}

int gpj_index_num_lines(const gpj_file* f, int64_t* lines) {
    if (!f || !lines) return GPJ_EINVAL;
    if (!f->indexed) return GPJ_ESTATE;
    *lines = f->num_lines;
    return GPJ_OK;
}

int gpj_index_copy_newlines(gpj_ctx* ctx, const gpj_file* f, int64_t* host, int64_t count) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_file(ctx, f))) return rc;
    if (!host) return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (!f->indexed) return fail(ctx, GPJ_ESTATE, "file is not indexed");
    if (count < f->num_lines) return fail(ctx, GPJ_EINVAL, "host buffer too small");
    GPJ_CUDA(ctx, cudaMemcpyAsync(host, f->d_nl, f->num_lines * 8, cudaMemcpyDeviceToHost, ctx->stream));
    GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GPJ_OK;
}

int gpj_index_copy_string_index(gpj_ctx* ctx, const gpj_file* f, uint64_t* host, int64_t count) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_file(ctx, f))) return rc;
    if (!host && f->words > 0) return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (!f->indexed) return fail(ctx, GPJ_ESTATE, "file is not indexed");
    if (count < f->words) return fail(ctx, GPJ_EINVAL, "host buffer too small");
    if (f->words == 0) return GPJ_OK;
    GPJ_CUDA(ctx, cudaMemcpyAsync(host, f->d_str, f->words * 8, cudaMemcpyDeviceToHost, ctx->stream));
    GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GPJ_OK;
}

int gpj_index_copy_leveled_bitmaps(gpj_ctx* ctx, const gpj_file* f, uint64_t* host, int64_t count) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_file(ctx, f))) return rc;
    if (!host && f->words > 0) return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (!f->indexed) return fail(ctx, GPJ_ESTATE, "file is not indexed");
    const int64_t total = f->words * f->num_levels;
    if (count < total) return fail(ctx, GPJ_EINVAL, "host buffer too small");
    if (total == 0) return GPJ_OK;
    GPJ_CUDA(ctx, cudaMemcpyAsync(host, f->d_lvl, total * 8, cudaMemcpyDeviceToHost, ctx->stream));
    GPJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GPJ_OK;
}

int gpj_build_index_device(gpj_ctx* ctx, const void* d_file, int64_t n, int num_levels,
                           uint64_t* d_string_index, uint64_t* d_leveled, int64_t* d_newlines,
                           int64_t newline_cap, int64_t* num_lines) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n < 0 || !num_lines || (n > 0 && (!d_file || !d_string_index || !d_leveled)) ||
        newline_cap < 0 || (newline_cap > 0 && !d_newlines))
        return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (reinterpret_cast<uintptr_t>(d_file) % 16 != 0)
        return fail(ctx, GPJ_EINVAL, "device input must be 16-byte aligned");
    if (num_levels < 1 || num_levels > GPJ_MAX_LEVELS)
        return fail(ctx, GPJ_ELIMIT, "Invalid number of levels: " + std::to_string(num_levels));
    const double t0 = now_ms();
    GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    rc = run_index(ctx, static_cast<const uint8_t*>(d_file), n, num_levels, d_string_index, d_leveled,
                   d_newlines, newline_cap, num_lines);
    if (rc) return rc;
    rc = end_phase(ctx, "build_index", t0);
    if (rc) return rc;
    if (*num_lines > newline_cap)
        return fail(ctx, GPJ_ELIMIT, "newline index needs " + std::to_string(*num_lines) + " entries");
    return GPJ_OK;
}

int gpj_query(gpj_ctx* ctx, gpj_file* f, int nq, const uint8_t* const* bc, const size_t* len,
              int slots, int64_t* host_out, int64_t out_count) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_file(ctx, f))) return rc;
    if (!bc || !len || !host_out) return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (f->indexed) {
        rc = ensure_out(ctx, f, static_cast<size_t>(std::max(nq, 1)) * f->num_lines * std::max(slots, 1) * 2);
        if (rc) return rc;
    }
    return query_common(ctx, f, nq, bc, len, slots, f->d_out, out_count, true, host_out);
}

int gpj_query_device(gpj_ctx* ctx, gpj_file* f, int nq, const uint8_t* const* bc, const size_t* len,
                     int slots, int64_t* d_out, int64_t out_count) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_file(ctx, f))) return rc;
    if (!bc || !len || !d_out) return fail(ctx, GPJ_EINVAL, "bad arguments");
    return query_common(ctx, f, nq, bc, len, slots, d_out, out_count, false, nullptr);
}

int gpj_index_query_device(gpj_ctx* ctx, gpj_file* f, int num_levels, int nq, const uint8_t* const* bc,
                           const size_t* len, int slots, int64_t* d_out, int64_t out_lines) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!f || f->ctx != ctx || !bc || !len || !d_out || out_lines < 1) return fail(ctx, GPJ_EINVAL, "bad arguments");
    return index_and_query(ctx, f, num_levels, nq, bc, len, slots, d_out, out_lines, nullptr);
}

// gpj_query_paths up to the results in f->d_out: [nq][*cap][*slots][2].
static int run_paths(gpj_ctx* ctx, gpj_file* f, int nq, const char* const* paths, int* slots_out,
                     int64_t* cap_out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_file(ctx, f))) return rc;
    if (!paths) return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (nq > GPJ_MAX_QUERIES) return fail(ctx, GPJ_ELIMIT, "Maximum size of queries is 255");
    if (nq < 1) return fail(ctx, GPJ_EINVAL, "expected queries to contain at least one query");
    std::vector<gpj::CompiledPath> compiled(static_cast<size_t>(nq));
    int depth = 0, slots = 0;
    for (int i = 0; i < nq; i++) {
        try {
            compiled[i] = gpj::compile_path(paths[i] ? paths[i] : "", ctx->path_extensions);
        } catch (const gpj::PathError& e) {
            if (e.unsupported)
                return fail(ctx, GPJ_EUNSUPPORTED, "Unsupported JSON path (" + std::to_string(i) + "): " + e.what());
            return fail(ctx, GPJ_EPARSE, "Failed to parse JSON path (" + std::to_string(i) + "): " + e.what());
        }
        depth = std::max(depth, compiled[i].max_depth);
        slots = std::max(slots, compiled[i].num_results);
    }
    if (depth > GPJ_MAX_LEVELS)
        return fail(ctx, GPJ_ELIMIT, "Invalid number of levels: " + std::to_string(depth));
    std::vector<const uint8_t*> bcs(static_cast<size_t>(nq));
    std::vector<size_t> lens(static_cast<size_t>(nq));
    for (int i = 0; i < nq; i++) {
        bcs[i] = compiled[i].bytecode.data();
        lens[i] = compiled[i].bytecode.size();
    }
    if (f->indexed && f->num_levels >= depth) {
        // the resident index has enough levels: the queries alone
        rc = ensure_out(ctx, f, static_cast<size_t>(nq) * f->num_lines * slots * 2);
        if (!rc) rc = query_common(ctx, f, nq, bcs.data(), lens.data(), slots, f->d_out,
                                   static_cast<int64_t>(nq) * f->num_lines * slots * 2, false, nullptr);
        if (!rc) rc = end_phase(ctx, "find_value", now_ms());
        if (rc) return rc;
        *slots_out = slots;
        *cap_out = f->num_lines;
        return GPJ_OK;
    }
    // One pass for index and queries, with results strided by a line
    // capacity (the newline-index estimate).
    int64_t cap = std::min<int64_t>(f->n + 1, f->n / 256 + 1024);
    for (int attempt = 0; attempt < 2; attempt++) {
        rc = ensure_out(ctx, f, static_cast<size_t>(nq) * cap * slots * 2);
        if (rc) return rc;
        int64_t needed = 0;
        rc = index_and_query(ctx, f, depth, nq, bcs.data(), lens.data(), slots, f->d_out, cap, &needed);
        if (rc == GPJ_ELIMIT && needed > cap) {
            cap = needed;
            continue;
        }
        break;
    }
    if (rc) return rc;
    *slots_out = slots;
    *cap_out = cap;
    return GPJ_OK;
}

int gpj_query_paths(gpj_ctx* ctx, gpj_file* f, int nq, const char* const* paths, gpj_result** out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out) return fail(ctx, GPJ_EINVAL, "bad arguments");
    int slots = 0;
    int64_t cap = 0;
    rc = run_paths(ctx, f, nq, paths, &slots, &cap);
    if (rc) return rc;
    gpj_result* r = new (std::nothrow) gpj_result;
    if (!r) return fail(ctx, GPJ_ENOMEM, "out of host memory");
    r->nq = nq;
    r->lines = f->num_lines;
    r->slots = slots;
    const size_t per_query = static_cast<size_t>(f->num_lines) * slots * 2;
    if (!r->allocate(static_cast<size_t>(nq) * per_query)) {
        delete r;
        return fail(ctx, GPJ_ENOMEM, "out of host memory for results");
    }
    const double t1 = now_ms();
    cudaEventRecord(ctx->ev0, ctx->stream);
    for (int q = 0; q < nq; q++) {
        cudaError_t e = cudaMemcpyAsync(r->offsets + q * per_query, f->d_out + static_cast<size_t>(q) * cap * slots * 2,
                                        per_query * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e != cudaSuccess) {
            delete r;
            return cuda_fail(ctx, e, "cudaMemcpyAsync(results)");
        }
    }
    rc = end_phase(ctx, "copy_results", t1);
    if (rc) {
        delete r;
        return rc;
    }
    *out = r;
    return GPJ_OK;
}

int64_t gpj_result_num_queries(const gpj_result* r) { return r ? r->nq : -1; }
int64_t gpj_result_num_lines(const gpj_result* r) { return r ? r->lines : -1; }
int gpj_result_slots(const gpj_result* r) { return r ? r->slots : -1; }
const int64_t* gpj_result_offsets(const gpj_result* r) { return r ? r->offsets : nullptr; }
void gpj_result_release(gpj_result* r) { delete r; }

int gpj_values_device(gpj_ctx* ctx, gpj_file* f, const int64_t* d_pairs, int64_t npairs, uint8_t* d_kinds,
                      int64_t* d_offsets, uint8_t* d_bytes, int64_t bytes_cap, int64_t* total_bytes) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_file(ctx, f))) return rc;
    if (npairs < 0 || (npairs > 0 && (!d_pairs || !d_kinds)) || !d_offsets || bytes_cap < 0 ||
        (bytes_cap > 0 && !d_bytes) || !total_bytes)
        return fail(ctx, GPJ_EINVAL, "bad arguments");
    const double t0 = now_ms();
    GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    // with bytes_cap 0 the copy kernel writes no byte, so d_bytes may be null
    rc = gather_values(ctx, f, d_pairs, npairs, npairs, npairs, d_kinds, d_offsets, bytes_cap > 0 ? d_bytes : nullptr,
                       bytes_cap, nullptr, total_bytes);
    if (rc) return rc;
    rc = end_phase(ctx, "gather_values", t0);
    if (rc) return rc;
    if (*total_bytes > bytes_cap)
        return fail(ctx, GPJ_ELIMIT, "values take " + std::to_string(*total_bytes) + " bytes, the buffer holds " +
                                         std::to_string(bytes_cap));
    return GPJ_OK;
}

int gpj_query_values(gpj_ctx* ctx, gpj_file* f, int nq, const char* const* paths, gpj_values** out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out) return fail(ctx, GPJ_EINVAL, "bad arguments");
    int slots = 0;
    int64_t cap = 0;
    rc = run_paths(ctx, f, nq, paths, &slots, &cap);
    if (rc) return rc;
    gpj_values* v = new (std::nothrow) gpj_values;
    if (!v) return fail(ctx, GPJ_ENOMEM, "out of host memory");
    v->nq = nq;
    v->lines = f->num_lines;
    v->slots = slots;
    const int64_t per_query = f->num_lines * slots;
    const int64_t npairs = per_query * nq;
    uint8_t* d_kinds = nullptr;
    int64_t* d_offsets = nullptr;
    uint8_t* d_bytes = nullptr;
    int64_t total = 0;
    const double t0 = now_ms();
    cudaEventRecord(ctx->ev0, ctx->stream);
    rc = device_alloc(ctx, &d_kinds, static_cast<size_t>(std::max<int64_t>(npairs, 1)), "cudaMalloc(value kinds)");
    if (!rc) rc = device_alloc(ctx, &d_offsets, static_cast<size_t>(npairs + 1), "cudaMalloc(value offsets)");
    if (!rc)
        rc = gather_values(ctx, f, f->d_out, npairs, per_query, cap * slots, d_kinds, d_offsets, nullptr, 0, &d_bytes,
                           &total);
    if (!rc) {
        try {
            v->kinds.resize(static_cast<size_t>(npairs));
            v->offsets.resize(static_cast<size_t>(npairs + 1));
            v->bytes.resize(static_cast<size_t>(total));
        } catch (const std::bad_alloc&) {
            rc = fail(ctx, GPJ_ENOMEM, "out of host memory for values");
        }
    }
    cudaError_t e = cudaSuccess;
    if (!rc && npairs > 0) e = cudaMemcpyAsync(v->kinds.data(), d_kinds, npairs, cudaMemcpyDeviceToHost, ctx->stream);
    if (!rc && e == cudaSuccess)
        e = cudaMemcpyAsync(v->offsets.data(), d_offsets, (npairs + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (!rc && e == cudaSuccess && total > 0)
        e = cudaMemcpyAsync(v->bytes.data(), d_bytes, total, cudaMemcpyDeviceToHost, ctx->stream);
    if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, "copy of values");
    device_free(ctx, d_kinds);
    device_free(ctx, d_offsets);
    device_free(ctx, d_bytes);
    if (!rc) rc = end_phase(ctx, "gather_values", t0);
    if (rc) {
        delete v;
        return rc;
    }
    *out = v;
    return GPJ_OK;
}

int64_t gpj_values_num_queries(const gpj_values* v) { return v ? v->nq : 0; }
int64_t gpj_values_num_lines(const gpj_values* v) { return v ? v->lines : 0; }
int gpj_values_slots(const gpj_values* v) { return v ? v->slots : 0; }
const uint8_t* gpj_values_kinds(const gpj_values* v) { return v ? v->kinds.data() : nullptr; }
const int64_t* gpj_values_offsets(const gpj_values* v) { return v ? v->offsets.data() : nullptr; }
const uint8_t* gpj_values_bytes(const gpj_values* v) { return v ? v->bytes.data() : nullptr; }
int64_t gpj_values_size(const gpj_values* v) { return v ? static_cast<int64_t>(v->bytes.size()) : 0; }
void gpj_values_release(gpj_values* v) { delete v; }

int gpj_get_timings(gpj_ctx* ctx, char* json, size_t cap, size_t* len) {
    if (!ctx) return GPJ_EINVAL;
    std::string s = "{\"phases\":[";
    for (size_t i = 0; i < ctx->phases.size(); i++) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "%s{\"name\":\"%s\",\"device_ms\":%.6f,\"host_ms\":%.6f}", i ? "," : "",
                      ctx->phases[i].name.c_str(), ctx->phases[i].device_ms, ctx->phases[i].host_ms);
        s += buf;
    }
    s += "],\"kernel_launches\":" + std::to_string(ctx->launches) +
         ",\"exact_index_fallbacks\":" + std::to_string(ctx->exact_fallbacks) + "}";
    if (len) *len = s.size();
    if (json && cap > 0) {
        const size_t k = std::min(cap - 1, s.size());
        std::memcpy(json, s.data(), k);
        json[k] = '\0';
    }
    return GPJ_OK;
}

void gpj_reset_timings(gpj_ctx* ctx) {
    if (ctx) ctx->phases.clear();
}

int64_t gpj_kernel_launches(const gpj_ctx* ctx) { return ctx ? ctx->launches : -1; }

}  // extern "C"

// ---- batches ---------------------------------------------------------------------

namespace {

// Indexes the batch's files whose resident index is missing or too shallow:
// one standalone index launch over all their tiles, one newline pass, one
// status read-back.  Files the batch launch cannot index (not line-delimited,
// a line longer than the look-ahead allows, more lines than estimated) are
// indexed again alone.
int batch_index(gpj_ctx* ctx, std::vector<gpj_batch::FileRun>& files) {
    std::vector<gpj_file*> need;
    int levels = 1;
    for (auto& fr : files) {
        gpj_file* f = fr.file;
        if (!f->indexed || f->num_levels < fr.depth) {
            need.push_back(f);
            levels = std::max(levels, fr.depth);
        }
    }
    if (need.empty()) return GPJ_OK;
    const double t0 = now_ms();
    GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    std::vector<gpj::TileFile> tf;
    std::vector<gpj::LineFile> lf;
    std::vector<gpj_file*> batched;
    int64_t total_tiles = 0, total_words = 0;
    int rc = GPJ_OK;
    for (gpj_file* f : need) {
        // a file of another context may still be in use on that context's
        // stream: wait for it before its index buffers are reallocated here
        if (f->ctx != ctx) GPJ_CUDA(ctx, cudaStreamSynchronize(f->ctx->stream));
        if ((rc = ensure_index_buffers(ctx, f, levels))) return rc;
        f->indexed = false;
        f->colon_valid = false;
        if (f->n == 0) continue;  // indexed alone below
        batched.push_back(f);
        total_tiles += (f->n + gpj::kStandaloneTileBytes - 1) / gpj::kStandaloneTileBytes;
        total_words += f->words;
    }
    const int nb = static_cast<int>(batched.size());
    if (nb > 0) {
        uint64_t* bits = nullptr;
        int32_t* counts = nullptr;
        int64_t* offsets = nullptr;
        unsigned long long* status = nullptr;
        gpj::TileFile* d_tf = nullptr;
        gpj::LineFile* d_lf = nullptr;
        rc = device_alloc(ctx, &bits, static_cast<size_t>(total_words), "cudaMalloc(batch newline bitmaps)");
        if (!rc) rc = device_alloc(ctx, &counts, static_cast<size_t>(total_tiles), "cudaMalloc(batch tile counts)");
        if (!rc)
            rc = device_alloc(ctx, &offsets, static_cast<size_t>(gpj::newline_offsets_words(total_tiles)),
                              "cudaMalloc(batch tile offsets)");
        if (!rc) rc = device_alloc(ctx, &status, static_cast<size_t>(2 * nb), "cudaMalloc(batch status)");
        if (!rc) rc = device_alloc(ctx, &d_tf, static_cast<size_t>(nb), "cudaMalloc(batch files)");
        if (!rc) rc = device_alloc(ctx, &d_lf, static_cast<size_t>(nb), "cudaMalloc(batch line files)");
        std::vector<unsigned long long> h_status(2 * static_cast<size_t>(nb));
        if (!rc) {
            int64_t tile = 0, word = 0;
            for (int i = 0; i < nb; i++) {
                gpj_file* f = batched[i];
                const int64_t ntiles = (f->n + gpj::kStandaloneTileBytes - 1) / gpj::kStandaloneTileBytes;
                tf.push_back(gpj::TileFile{f->d_data, f->n, f->n, f->d_str, f->d_lvl, f->words, bits + word,
                                           status + 2 * i, tile, f->d_colon});
                lf.push_back(gpj::LineFile{bits + word, f->words, f->d_nl, f->nl_cap, status + 2 * i, tile, ntiles});
                tile += ntiles;
                word += f->words;
            }
            cudaError_t e = cudaMemsetAsync(status, 0, 2 * sizeof(unsigned long long) * nb, ctx->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_status, 0, 2 * sizeof(unsigned long long), ctx->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d_tf, tf.data(), sizeof(gpj::TileFile) * nb, cudaMemcpyHostToDevice, ctx->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d_lf, lf.data(), sizeof(gpj::LineFile) * nb, cudaMemcpyHostToDevice, ctx->stream);
            if (e == cudaSuccess) {
                gpj::IndexParams p{};
                p.num_levels = levels;
                p.materialize = 1;
                p.tile_begin = 0;
                p.tile_end = total_tiles;
                p.batch = d_tf;
                p.batch_files = nb;
                // a file of a batch is small (its long lines cost one CTA
                // little) and its re-indexing alone would cost a launch
                // and a wait: lines up to 8 MiB past a tile stay in the launch
                p.max_extension = kBatchMaxExtension;
                p.status = ctx->d_status;
                p.tile_newlines = counts;
                const int occ = tile_ctas_per_sm(ctx, levels);
                const int64_t grid = std::min<int64_t>(total_tiles, static_cast<int64_t>(ctx->sms) * occ);
                p.tile_counter = tile_claims(ctx);
                e = cudaMemsetAsync(p.tile_counter, 0, sizeof(unsigned int), ctx->stream);
                if (e == cudaSuccess) e = gpj::launch_tile_index_kernel(p, static_cast<int>(grid), ctx->stream);
                ctx->launches++;
            }
            if (e == cudaSuccess) {
                const int64_t grid = std::min<int64_t>((total_tiles + 7) / 8, static_cast<int64_t>(ctx->sms) * 8);
                e = gpj::launch_newline_index_batch(counts, total_tiles, d_lf, nb, offsets, static_cast<int>(grid),
                                                    ctx->stream);
                ctx->launches += 2;
            }
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(h_status.data(), status, 2 * sizeof(unsigned long long) * nb,
                                    cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(ctx->h_status, ctx->d_status, 2 * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batch index");
        }
        device_free(ctx, bits);
        device_free(ctx, counts);
        device_free(ctx, offsets);
        device_free(ctx, status);
        device_free(ctx, d_tf);
        device_free(ctx, d_lf);
        if (rc) return rc;
        if ((rc = status_error(ctx, ctx->h_status[1]))) return rc;
        for (int i = 0; i < nb; i++) {
            gpj_file* f = batched[i];
            const unsigned long long errs = h_status[2 * i + 1];
            const int64_t lines = static_cast<int64_t>(h_status[2 * i]);
            if ((errs & (gpj::kErrIrregular | gpj::kErrLongLine)) || lines > f->nl_cap) continue;  // alone below
            if ((rc = status_error(ctx, errs))) return rc;
            f->num_lines = lines;
            f->num_levels = levels;
            f->indexed = true;
            f->colon_valid = true;
        }
    }
    for (gpj_file* f : need)
        if (!f->indexed && (rc = index_pass(ctx, f, levels, nullptr, nullptr))) return rc;
    return end_phase(ctx, "batch_index", t0);
}

}  // namespace

extern "C" {

int gpj_batch_create(gpj_ctx* ctx, gpj_batch** out) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out) return fail(ctx, GPJ_EINVAL, "bad arguments");
    gpj_batch* b = new (std::nothrow) gpj_batch;
    if (!b) return fail(ctx, GPJ_ENOMEM, "out of host memory");
    b->ctx = ctx;
    *out = b;
    return GPJ_OK;
}

int gpj_batch_add(gpj_batch* b, gpj_file* f, int nq, const char* const* paths, int* item) {
    if (!b) return GPJ_EINVAL;
    gpj_ctx* ctx = b->ctx;
    if (!f || !paths || nq < 1 || !item) return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (nq > GPJ_MAX_QUERIES) return fail(ctx, GPJ_ELIMIT, "Maximum size of queries is 255");
    int dev = -1;
    if (f->ctx) dev = f->ctx->device;
    if (dev != ctx->device) return fail(ctx, GPJ_EINVAL, "file is on another device");
    gpj_batch::Item it;
    it.file = f;
    for (int i = 0; i < nq; i++) {
        try {
            it.queries.push_back(gpj::compile_path(paths[i] ? paths[i] : "", ctx->path_extensions));
        } catch (const gpj::PathError& e) {
            if (e.unsupported)
                return fail(ctx, GPJ_EUNSUPPORTED, "Unsupported JSON path (" + std::to_string(i) + "): " + e.what());
            return fail(ctx, GPJ_EPARSE, "Failed to parse JSON path (" + std::to_string(i) + "): " + e.what());
        }
        if (it.queries.back().max_depth > GPJ_MAX_LEVELS)
            return fail(ctx, GPJ_ELIMIT, "Invalid number of levels: " + std::to_string(it.queries.back().max_depth));
    }
    b->items.push_back(std::move(it));
    b->ran = false;
    b->dirty = true;
    *item = static_cast<int>(b->items.size() - 1);
    return GPJ_OK;
}

int gpj_batch_run(gpj_batch* b) {
    if (!b) return GPJ_EINVAL;
    gpj_ctx* ctx = b->ctx;
    int rc = check_ctx(ctx);
    if (rc) return rc;
    b->files.clear();
    b->ran = false;
    for (auto& it : b->items) {
        int slot = -1;
        for (size_t i = 0; i < b->files.size(); i++)
            if (b->files[i].file == it.file) slot = static_cast<int>(i);
        if (slot < 0) {
            b->files.emplace_back();
            b->files.back().file = it.file;
            slot = static_cast<int>(b->files.size() - 1);
        }
        auto& fr = b->files[slot];
        it.file_slot = slot;
        it.q0 = static_cast<int>(fr.queries.size());
        for (auto& q : it.queries) {
            fr.queries.push_back(&q);
            fr.depth = std::max(fr.depth, q.max_depth);
            fr.slots = std::max(fr.slots, q.num_results);
        }
    }
    if (b->files.empty()) return GPJ_OK;
    if ((rc = batch_index(ctx, b->files))) return rc;

    // one find_value launch over every line of every file
    const double t0 = now_ms();
    GPJ_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    std::vector<uint8_t> blob;  // per file: [int32 offsets (16-byte padded)][bytecode]
    std::vector<size_t> blob_at(b->files.size());
    size_t total_out = 0;
    int64_t total_items = 0;
    for (size_t i = 0; i < b->files.size(); i++) {
        auto& fr = b->files[i];
        const size_t nq = fr.queries.size();
        blob_at[i] = blob.size();
        const size_t header = ((nq * 4 + 15) / 16) * 16;
        blob.resize(blob.size() + header, 0);
        size_t code = 0;
        for (size_t q = 0; q < nq; q++) {
            const int32_t off = static_cast<int32_t>(code);
            std::memcpy(blob.data() + blob_at[i] + 4 * q, &off, 4);
            blob.insert(blob.end(), fr.queries[q]->bytecode.begin(), fr.queries[q]->bytecode.end());
            code += fr.queries[q]->bytecode.size();
        }
        blob.resize((blob.size() + 15) / 16 * 16, 0);
        fr.lines = fr.file->num_lines;
        fr.out_offset = total_out;
        total_out += nq * static_cast<size_t>(fr.lines) * fr.slots * 2;
        total_items += gpj::query_items(fr.lines, static_cast<int>(nq));
    }
    // what the query phase reads: replay its graph when nothing of it changed
    int depth = 0;
    for (auto& fr : b->files) depth = std::max(depth, fr.depth);
    std::vector<uint64_t> sig{static_cast<uint64_t>(reinterpret_cast<uintptr_t>(ctx->stream)),
                              static_cast<uint64_t>(ctx->tuning.long_line_bytes),
                              static_cast<uint64_t>(query_occupancy(ctx, depth))};
    for (auto& fr : b->files) {
        gpj_file* f = fr.file;
        for (uint64_t v : {static_cast<uint64_t>(reinterpret_cast<uintptr_t>(f)),
                           static_cast<uint64_t>(reinterpret_cast<uintptr_t>(f->d_data)),
                           static_cast<uint64_t>(reinterpret_cast<uintptr_t>(f->d_nl)),
                           static_cast<uint64_t>(reinterpret_cast<uintptr_t>(f->d_str)),
                           static_cast<uint64_t>(reinterpret_cast<uintptr_t>(f->d_lvl)),
                           static_cast<uint64_t>(reinterpret_cast<uintptr_t>(f->colon_valid ? f->d_colon : nullptr)),
                           static_cast<uint64_t>(f->num_lines), static_cast<uint64_t>(f->n)})
            sig.push_back(v);
    }
    if (!b->dirty && b->replay.exec && b->replay.sig == sig && b->replay.dst->refs.load() == 1) {
        cudaError_t e = cudaGraphLaunch(b->replay.exec, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "batch query (graph)");
        ctx->launches += long_lines(ctx).items ? 2 : 1;
        b->cur = b->replay.dst;
        b->replays++;
        rc = end_phase(ctx, "batch_query_replay", t0);
        if (rc) return rc;
        b->ran = true;
        return GPJ_OK;
    }
    b->drop_replay();
    // a graph pays off from the third identical run on: capture only when
    // the requests did not change since the last run (a serving loop's
    // batches, new every time, run directly)
    const bool try_capture = !b->dirty;
    b->dirty = false;
    uint8_t* d_blob = nullptr;
    int64_t* d_out = nullptr;
    gpj::QueryFile* d_qf = nullptr;
    rc = device_alloc(ctx, &d_blob, blob.size(), "cudaMalloc(batch bytecode)");
    if (!rc) rc = device_alloc(ctx, &d_out, std::max<size_t>(total_out, 1), "cudaMalloc(batch results)");
    if (!rc) rc = device_alloc(ctx, &d_qf, b->files.size(), "cudaMalloc(batch query files)");
    bool captured = false;
    if (!rc) {
        std::vector<gpj::QueryFile> qf;
        int64_t item = 0;
        for (size_t i = 0; i < b->files.size(); i++) {
            auto& fr = b->files[i];
            gpj_file* f = fr.file;
            const size_t nq = fr.queries.size();
            const size_t header = ((nq * 4 + 15) / 16) * 16;
            qf.push_back(gpj::QueryFile{f->d_data, f->n, f->d_nl, fr.lines, f->d_str, f->d_lvl, f->words,
                                        d_blob + blob_at[i] + header,
                                        reinterpret_cast<const int32_t*>(d_blob + blob_at[i]),
                                        static_cast<int>(nq), fr.slots, d_out + fr.out_offset, fr.lines, item,
                                        f->colon_valid ? f->d_colon : nullptr});
            item += gpj::query_items(fr.lines, static_cast<int>(nq));
        }
        cudaError_t e = cudaMemcpyAsync(d_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_qf, qf.data(), sizeof(gpj::QueryFile) * qf.size(), cudaMemcpyHostToDevice,
                                ctx->stream);
        // a page-locked buffer no result of an earlier run refers to (every
        // earlier run's copy has completed: each run ends synchronised)
        PinnedResults* pick = nullptr;
        for (PinnedResults* r : b->pool)
            if (!pick && r->refs.load() == 1 && r->cap >= std::max<size_t>(total_out, 1)) pick = r;
        if (e == cudaSuccess && !pick) {
            // drop the idle buffers (too small), then allocate with a quarter to spare
            std::vector<PinnedResults*> keep;
            for (PinnedResults* r : b->pool) {
                if (r->refs.load() == 1)
                    unref(r);
                else
                    keep.push_back(r);
            }
            b->pool.swap(keep);
            PinnedResults* r = new (std::nothrow) PinnedResults;
            if (!r) {
                e = cudaErrorMemoryAllocation;
            } else {
                const size_t cap = std::max<size_t>(total_out + total_out / 4, 1 << 16);
                e = cudaMallocHost(&r->p, cap * 8);
                if (e == cudaSuccess) {
                    r->cap = cap;
                    b->pool.push_back(r);
                    pick = r;
                } else {
                    delete r;
                }
            }
        }
        if (pick) b->cur = pick;
        // the query phase: captured as a graph (kept for the next run) when
        // the stream allows it, else launched directly
        const int64_t grid = std::max<int64_t>(
            1, std::min<int64_t>((total_items + gpj::kQueryThreads - 1) / gpj::kQueryThreads,
                                 static_cast<int64_t>(ctx->sms) * query_occupancy(ctx, depth)));
        const gpj::LongLines ll = long_lines(ctx);
        auto query_phase = [&]() -> cudaError_t {
            cudaError_t q = cudaSuccess;
            if (total_items > 0) {
                if (ll.items) q = cudaMemsetAsync(ctx->d_long_count, 0, sizeof(unsigned long long), ctx->stream);
                if (q == cudaSuccess)
                    q = gpj::launch_find_value_batch(d_qf, static_cast<int>(qf.size()), total_items, depth, ll,
                                                     static_cast<int>(grid), ctx->sms * 2, ctx->stream);
            }
            if (q == cudaSuccess && total_out > 0)
                q = cudaMemcpyAsync(pick->p, d_out, total_out * 8, cudaMemcpyDeviceToHost, ctx->stream);
            return q;
        };
        cudaGraphExec_t exec = nullptr;
        if (e == cudaSuccess) {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            cudaError_t ce = cudaStreamIsCapturing(ctx->stream, &cs);
            if (try_capture && ce == cudaSuccess && cs == cudaStreamCaptureStatusNone && ctx->stream != nullptr &&
                cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                const cudaError_t qe = query_phase();
                cudaGraph_t graph = nullptr;
                const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &graph);
                if (qe == cudaSuccess && ee == cudaSuccess && graph &&
                    cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
                    captured = true;
                } else {
                    exec = nullptr;
                }
                if (graph) cudaGraphDestroy(graph);
                cudaGetLastError();
            }
            e = captured ? cudaGraphLaunch(exec, ctx->stream) : query_phase();
        }
        ctx->launches += ll.items ? 2 : 1;
        if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, "batch query");
        if (captured && !rc) {
            b->replay.exec = exec;
            b->replay.sig = sig;
            b->replay.d_blob = d_blob;
            b->replay.d_out = d_out;
            b->replay.d_qf = d_qf;
            b->replay.dst = pick;  // a buffer of the pool: replayed only while no result refers to it
            b->replay.stream = ctx->stream;
        } else if (exec) {
            cudaGraphExecDestroy(exec);
            captured = false;
        }
    }
    if (!captured) {
        device_free(ctx, d_blob);
        device_free(ctx, d_out);
        device_free(ctx, d_qf);
    }
    if (rc) return rc;
    rc = end_phase(ctx, "batch_query", t0);
    if (rc) return rc;
    b->ran = true;
    return GPJ_OK;
}

int gpj_batch_result(gpj_batch* b, int item, gpj_result** out) { return gpj_batch_result_ex(b, item, 0, out); }

int gpj_batch_result_ex(gpj_batch* b, int item, int slots, gpj_result** out) {
    if (!b) return GPJ_EINVAL;
    gpj_ctx* ctx = b->ctx;
    if (!out || item < 0 || item >= static_cast<int>(b->items.size()) || slots < 0)
        return fail(ctx, GPJ_EINVAL, "bad arguments");
    if (!b->ran) return fail(ctx, GPJ_ESTATE, "batch has not run since its last change");
    const auto& it = b->items[item];
    const auto& fr = b->files[it.file_slot];
    if (slots > fr.slots) return fail(ctx, GPJ_EINVAL, "more slots than the batch has for the file");
    if (slots == 0) slots = fr.slots;
    gpj_result* r = new (std::nothrow) gpj_result;
    if (!r) return fail(ctx, GPJ_ENOMEM, "out of host memory");
    r->nq = static_cast<int64_t>(it.queries.size());
    r->lines = fr.lines;
    r->slots = slots;
    const size_t per_query = static_cast<size_t>(fr.lines) * fr.slots * 2;
    int64_t* src = b->cur->p + fr.out_offset + it.q0 * per_query;
    if (slots == fr.slots) {
        // a view of the run's page-locked results, kept alive by the view
        b->cur->refs.fetch_add(1);
        r->backing = b->cur;
        r->offsets = src;
        *out = r;
        return GPJ_OK;
    }
    if (!r->allocate(static_cast<size_t>(r->nq) * fr.lines * slots * 2)) {
        delete r;
        return fail(ctx, GPJ_ENOMEM, "out of host memory for results");
    }
    {  // each line's first `slots` pairs
        const size_t lines = static_cast<size_t>(r->nq) * fr.lines;
        for (size_t l = 0; l < lines; l++)
            std::memcpy(r->offsets + l * slots * 2, src + l * fr.slots * 2, static_cast<size_t>(slots) * 2 * 8);
    }
    *out = r;
    return GPJ_OK;
}

int gpj_batch_size(const gpj_batch* b) { return b ? static_cast<int>(b->items.size()) : -1; }

void gpj_batch_clear(gpj_batch* b) {
    if (!b) return;
    b->items.clear();
    b->files.clear();
    b->ran = false;
    b->dirty = true;
}

void gpj_batch_release(gpj_batch* b) { delete b; }

}  // extern "C"
