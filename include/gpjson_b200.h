/*
 * gpjson_b200.h — C ABI of the B200-native GPJSON structural-index and
 * JSONPath query path.
 *
 * This library replaces the layer under GPJSON's `query(file, jsonpath)`
 * (gpjson/src/main/java/com/koenv/gpjson/functions/QueryFunction.java:48-265):
 * the grCUDA-derived runtime that reached libcudart/libcuda/libnvrtc through
 * Truffle NFI (gpu/CUDARuntime.java:76-94, gpu/CUDARuntimeFunction.java:39-186),
 * the index stages with their host-side carry scans (stages/CombinedIndex.java,
 * stages/LeveledBitmapsIndex.java) and the per-query find_value launches.
 * A Java caller binds these symbols with the Panama FFM API; Python binds them
 * with ctypes (gpjson_b200/_lib.py).
 *
 * Conventions
 *  - Every function returning int returns GPJ_OK (0) or a negative GPJ_E*
 *    code and never aborts the process.  The message of the last failure on a
 *    context is available from gpj_last_error().
 *  - Offsets are int64; -1 marks a miss (QueryFunction.java:197).
 *  - Host output buffers are owned by the caller; device buffers are owned by
 *    the gpj_file they belong to, except where a function takes device
 *    pointers explicitly.
 *  - A gpj_file is used with the context that made it; the other contexts'
 *    entry points refuse it with GPJ_EINVAL (gpj_batch_add alone takes
 *    files of other contexts on the same device).
 *  - One gpj_ctx must not be used by two threads at the same time.
 *  - All device work of a context runs on one CUDA stream (gpj_set_stream).
 */
#ifndef GPJSON_B200_H
#define GPJSON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Exported even when the library is built with -fvisibility=hidden. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- status codes ------------------------------------------------------ */
#define GPJ_OK 0
#define GPJ_EINVAL (-1)       /* bad argument: null pointer, size, alignment */
#define GPJ_EPARSE (-2)       /* JSONPathException (jsonpath/JSONPathException.java) */
#define GPJ_EUNSUPPORTED (-3) /* UnsupportedJSONPathException; GPJSON would fall back to
                                 Jayway JsonPath on the CPU (QueryFunction.java:122-128),
                                 which this library does not provide */
#define GPJ_ECUDA (-4)        /* a CUDA runtime call failed (GPJSONException.java:33-39) */
#define GPJ_ENOMEM (-5)       /* device or pinned-host allocation failed */
#define GPJ_EIO (-6)          /* the input file could not be opened or read */
#define GPJ_ELIMIT (-7)       /* a documented limit was exceeded */
#define GPJ_EDEVICE (-8)      /* a kernel reported an error word (bounded wait expired) */
#define GPJ_ESTATE (-9)       /* object not in the state the call needs */
#define GPJ_EAGAIN (-10)      /* not finished yet (gpj_serve_poll) */

/* Limits kept from the reference. */
#define GPJ_MAX_QUERIES 255   /* QueryFunction.java:74-77 */
#define GPJ_MAX_LEVELS 16     /* LeveledBitmapsIndex.java:16,31-33 */

typedef struct gpj_ctx gpj_ctx;
typedef struct gpj_file gpj_file;
typedef struct gpj_result gpj_result;
typedef struct gpj_values gpj_values;

/* ---- context ------------------------------------------------------------ */

/* Creates a context on CUDA device `device` (GPJSONContext.java:48-54 and the
 * CUDARuntime constructor, CUDARuntime.java:76-94).  Kernels are compiled
 * ahead of time for sm_100a, so there is no run-time NVRTC step
 * (CUDARuntime.java:267-289). */
int gpj_create(int device, gpj_ctx **out);
void gpj_destroy(gpj_ctx *ctx);

/* Message of the last failure on `ctx` (or of the last failed gpj_create when
 * ctx is NULL).  Valid until the next call on the same context. */
const char *gpj_last_error(const gpj_ctx *ctx);

/* Runs all later device work of `ctx` on `stream` (a cudaStream_t; NULL =
 * the context's own stream).  The reference runs everything synchronously on
 * the legacy default stream (CUDARuntime.java:388). */
int gpj_set_stream(gpj_ctx *ctx, void *stream);

/* Launch shapes of a context's kernels (no counterpart in the reference,
 * whose launch shapes are fixed: 8x1024 threads for the index kernels and
 * 512x1024 for find_value, stages/CombinedIndex.java:28-56,
 * functions/QueryFunction.java:201-241).  Results do not depend on them.
 *  - long_line_bytes: find_value evaluates lines longer than this with a
 *    whole warp each instead of one thread (0 = the default, 65536; -1 = never);
 *  - query_ctas_per_sm, index_ctas_per_sm: resident CTAs per SM of
 *    find_value and of the standalone index kernel (0 = the occupancy
 *    maximum; larger values are capped at it);
 *  - chunk_tiles: gpj_index_query_device and gpj_query_paths build the index
 *    and evaluate the queries chunk by chunk, chunks of this many 30 KiB
 *    tiles (a multiple of 1024), so that find_value reads each chunk's index
 *    from L2 right after it is written (0, the default = one index pass over
 *    the whole file, then one find_value pass; on tweet-like NDJSON the
 *    whole-file passes are faster, since find_value needs more lines than a
 *    chunk holds to hide its load latency);
 *  - reserved: 0.
 * gpjson_b200.tune (Python) measures and persists them per device. */
typedef struct gpj_tuning {
    int64_t long_line_bytes;
    int32_t query_ctas_per_sm;
    int32_t index_ctas_per_sm;
    int32_t chunk_tiles;
    int32_t reserved;
} gpj_tuning;

int gpj_set_tuning(gpj_ctx *ctx, const gpj_tuning *tuning);
int gpj_get_tuning(const gpj_ctx *ctx, gpj_tuning *out);

/* How gpj_index_query_device and gpj_query_paths evaluate queries: 0 (the
 * default) builds the index with one kernel and then evaluates all queries
 * with one find_value launch; 1 evaluates them inside the index kernel, on
 * the tile's masks in shared memory, where the input allows (well-formed
 * NDJSON, lines that fit a tile's look-ahead) and finishes the rest with
 * find_value.  Results are identical either way. */
int gpj_set_query_fusion(gpj_ctx *ctx, int enabled);

/* The JSONPath extensions (GPJ_PATH_* flags, default none) the calls that
 * take path strings compile with: gpj_query_paths, gpj_query_values,
 * gpj_batch_add. */
int gpj_set_path_extensions(gpj_ctx *ctx, unsigned extensions);

/* Library version string, e.g. "gpjson_b200 0.1 sm_100a". */
const char *gpj_version(void);

/* ---- JSONPath compiler --------------------------------------------------- */

/* Compiles `path` (NUL-terminated UTF-8) to GPJSON bytecode, byte-identical to
 * JSONPathParser.compile() (jsonpath/JSONPathParser.java:20-29).
 * On success writes the bytecode (at most `cap` bytes) to `out`, its length to
 * *len, JSONPathResult.getMaxDepth() to *max_depth and getNumResults() to
 * *num_results.  On GPJ_EPARSE / GPJ_EUNSUPPORTED a message is written to
 * `err` (at most err_cap bytes, NUL-terminated) when err is not NULL.
 * Returns GPJ_ELIMIT when the bytecode does not fit in `cap`. */
int gpj_compile(const char *path, uint8_t *out, size_t cap, size_t *len, int *max_depth,
                int *num_results, char *err, size_t err_cap);

/* JSONPath beyond the reference's subset, off by default: with no flag set,
 * paths are accepted and rejected exactly as the reference does (which
 * sends the others to its CPU fallback, JSONPathParser.java:84).
 * GPJ_PATH_INDEX_UNIONS: `[i,j,...]` with strictly ascending indices,
 * compiled like the reference's `[a:b]` ranges (one result slot per index,
 * each branch evaluating the rest of the path, with the ranges' behaviour
 * for index steps later in the path: their array's element counter carries
 * over from the previous branch); descending or repeated indices stay
 * GPJ_EUNSUPPORTED. */
#define GPJ_PATH_INDEX_UNIONS 1u

/* gpj_compile with the extensions in `extensions` (GPJ_PATH_* flags). */
int gpj_compile_ex(const char *path, unsigned extensions, uint8_t *out, size_t cap, size_t *len,
                   int *max_depth, int *num_results, char *err, size_t err_cap);

/* ---- input files ---------------------------------------------------------- */

/* Reads a whole NDJSON file into device memory (QueryFunction.readFile,
 * QueryFunction.java:316-335) through pinned staging buffers and async copies. */
int gpj_file_open(gpj_ctx *ctx, const char *filename, gpj_file **out);

/* Copies `n` bytes of host memory into device memory as an input file. */
int gpj_file_from_host(gpj_ctx *ctx, const void *data, int64_t n, gpj_file **out);

/* gpj_file_from_host followed by gpj_index_build, pipelined: the input is
 * copied in 56 MiB chunks on a second stream while the index kernel indexes
 * each chunk as soon as the chunk after it has arrived, so the copy and the
 * index build overlap (the reference reads and copies the whole file before
 * its first kernel, QueryFunction.java:316-335).  Same index as
 * gpj_index_build; inputs that are not line-delimited, or have lines longer
 * than a chunk, are indexed again once the copy is complete.  Page-locked
 * host memory gives the fastest copies. */
int gpj_file_from_host_indexed(gpj_ctx *ctx, const void *data, int64_t n, int num_levels,
                               gpj_file **out);

/* gpj_file_from_host_indexed and gpj_query in one pipelined call: while
 * the input is still being copied, each chunk's newline index is built right
 * after its index kernel and find_value runs on the lines it completes, so
 * the queries overlap the copy as well (the reference's query() reads the
 * file, then indexes it, then runs one find_value launch per query,
 * QueryFunction.java:165-241, one after the other).  Results as gpj_query:
 * int64[nq][lines][result_slots][2] into host_out (`out_count` elements;
 * page-locked memory copies fastest).  *num_lines receives the line count;
 * when host_out is too small the call returns GPJ_ELIMIT after indexing, with
 * *num_lines and *out set, and gpj_query on *out gives the results.  *out is
 * the indexed file (num_levels levels), to release with gpj_file_release. */
int gpj_file_from_host_query(gpj_ctx *ctx, const void *data, int64_t n, int num_levels, int nq,
                             const uint8_t *const *bytecode, const size_t *bytecode_len,
                             int result_slots, int64_t *host_out, int64_t out_count,
                             int64_t *num_lines, gpj_file **out);

/* Wraps `n` bytes that are already in device memory (not copied, not freed).
 * `d_data` must be 16-byte aligned and stay valid until gpj_file_release. */
int gpj_file_from_device(gpj_ctx *ctx, const void *d_data, int64_t n, gpj_file **out);

/* Frees the file's device buffers (input copy, index, results). */
void gpj_file_release(gpj_file *file);

int64_t gpj_file_size(const gpj_file *file);

/* ---- structural index ------------------------------------------------------ */

/* Builds the newline index, the string (in-string) bitmap and `num_levels`
 * leveled structural bitmaps of `file` in one pass over the input
 * (CombinedIndex.create, CombinedIndex.java:28-56, and
 * LeveledBitmapsIndex.create, LeveledBitmapsIndex.java:40-54, including their
 * host-side carry scans :98-115, :129-151 and :68-87, which run on the device
 * here).  1 <= num_levels <= GPJ_MAX_LEVELS.  Synchronous: on return the
 * index is complete and the line count is known. */
int gpj_index_build(gpj_ctx *ctx, gpj_file *file, int num_levels);

/* Number of lines = newline-index entries = '\n' count + 1. */
int gpj_index_num_lines(const gpj_file *file, int64_t *lines);

/* Copies the index to host memory: newline index (int64[lines]: [0]=0 then
 * every '\n' offset), string index (uint64[ceil(n/64)]) and leveled bitmaps
 * (uint64[num_levels][ceil(n/64)], level-major).  `count` is the number of
 * elements the host buffer holds; it must be at least the index size. */
int gpj_index_copy_newlines(gpj_ctx *ctx, const gpj_file *file, int64_t *host, int64_t count);
int gpj_index_copy_string_index(gpj_ctx *ctx, const gpj_file *file, uint64_t *host,
                                int64_t count);
int gpj_index_copy_leveled_bitmaps(gpj_ctx *ctx, const gpj_file *file, uint64_t *host,
                                   int64_t count);

/* Device-side stage entry: builds the same index from caller-owned device
 * buffers, the way the reference's stage tests drive CombinedIndex and
 * LeveledBitmapsIndex on raw device pointers (StringIndexTest.java,
 * NewlineIndexTest.java, LeveledBitmapsIndexTest.java).
 * d_file: n bytes, 16-byte aligned.  d_string_index: ceil(n/64) words.
 * d_leveled: num_levels*ceil(n/64) words.  d_newlines: newline_cap entries.
 * *num_lines receives the line count; when it exceeds newline_cap only the
 * first newline_cap entries were written and GPJ_ELIMIT is returned. */
int gpj_build_index_device(gpj_ctx *ctx, const void *d_file, int64_t n, int num_levels,
                           uint64_t *d_string_index, uint64_t *d_leveled, int64_t *d_newlines,
                           int64_t newline_cap, int64_t *num_lines);

/* Largest input gpj_build_index_device_noalloc accepts (256 MiB). */
#define GPJ_NOALLOC_MAX_BYTES (256LL << 20)

/* No counterpart in the reference (its stages allocate through
 * CUDARuntime/cudaMalloc on every call).  Same index as
 * gpj_build_index_device, same buffers and results, but it allocates no
 * memory, host or device, and needs no context: the kernels' scratch (tile
 * states, tile counter, status words) is one file-scope __device__ array of
 * about 384 KiB per device, sized for inputs of at most GPJ_NOALLOC_MAX_BYTES;
 * larger inputs return GPJ_ELIMIT before anything runs.
 * It works on the calling thread's current device and on `stream` (a
 * cudaStream_t of that device; NULL = the legacy default stream), and
 * synchronizes that stream before returning (to read the line count).
 * The first call on a device looks the array up (cudaGetSymbolAddress) and
 * sets the kernels' shared-memory attributes; make it before any
 * latency-critical call.  Every call reads its status back and waits for its
 * stream, so no call may be made on a stream that is being captured into a
 * graph (GPJ_EINVAL).  All calls on one device share the array, and calls
 * that overlapped on the GPU would race on it: within a process the library
 * serializes the calls on one device (a lock held until the call's device
 * work has finished), so a second thread's call waits for the first.
 * Returns GPJ_OK, GPJ_EINVAL, GPJ_ELIMIT (input too large or newline_cap too
 * small), GPJ_ECUDA (CUDA error or a device that is not sm_100) or
 * GPJ_EDEVICE (a kernel wait expired, in either pass).  There is no context
 * to carry a message; the code is the whole report. */
int gpj_build_index_device_noalloc(void *stream, const void *d_file, int64_t n, int num_levels,
                                   uint64_t *d_string_index, uint64_t *d_leveled,
                                   int64_t *d_newlines, int64_t newline_cap, int64_t *num_lines);

/* ---- queries ---------------------------------------------------------------- */

/* Evaluates `nq` compiled queries (bytecode from gpj_compile) over every line
 * of an indexed file in one pass, all queries of a line handled together.
 * Results are identical to running each query alone (the reference reuses
 * one result buffer across queries, QueryFunction.java:194-201, so lines a
 * later query misses keep an earlier query's offsets; this library does not).
 * `result_slots` must be at least every query's num_results; the output
 * layout is int64[nq][lines][result_slots][2] = (start, end) byte offsets,
 * -1 for a miss (find_value.cu result layout, QueryFunction.java:194).
 * The file must be indexed with at least max(max_depth) levels. */
int gpj_query(gpj_ctx *ctx, gpj_file *file, int nq, const uint8_t *const *bytecode,
              const size_t *bytecode_len, int result_slots, int64_t *host_out,
              int64_t out_count);

/* Same as gpj_query but writes the results to caller-owned device memory
 * `d_out` (same layout) and does not synchronise the stream. */
int gpj_query_device(gpj_ctx *ctx, gpj_file *file, int nq, const uint8_t *const *bytecode,
                     const size_t *bytecode_len, int result_slots, int64_t *d_out,
                     int64_t out_count);

/* Builds the index of `file` with `num_levels` levels and evaluates the `nq`
 * compiled queries in the same pass over the input: each line is indexed
 * and queried while its bytes and bitmaps are in shared memory (the
 * reference runs CombinedIndex, LeveledBitmapsIndex and one find_value
 * launch per query, QueryFunction.java:165-241).  The index is kept as by
 * gpj_index_build.  d_out: caller-owned device memory holding
 * int64[nq][out_lines][slots][2]; out_lines must be at least the file's line
 * count (GPJ_ELIMIT otherwise; the index is built and gpj_index_num_lines
 * reports the count).  Lines stay -1 where a query misses; results equal
 * running each query alone.  Synchronous. */
int gpj_index_query_device(gpj_ctx *ctx, gpj_file *file, int num_levels, int nq,
                           const uint8_t *const *bytecode, const size_t *bytecode_len,
                           int result_slots, int64_t *d_out, int64_t out_lines);

/* The whole reference call query(file, paths) (QueryFunction.call,
 * QueryFunction.java:48-265) on an opened file: compiles the paths, builds
 * the index with max(max_depth) levels (reusing an index that has enough
 * levels), runs all queries in one pass and copies the offsets to the host.
 * Path errors return GPJ_EPARSE ("Failed to parse JSON path (i)") or
 * GPJ_EUNSUPPORTED ("Unsupported JSON path (i)"). */
int gpj_query_paths(gpj_ctx *ctx, gpj_file *file, int nq, const char *const *paths,
                    gpj_result **out);

/* Result of gpj_query_paths: the Result/ResultArray/ResultItem layout
 * (result/Result.java:23-29): [query][line][slot] -> (start, end). */
int64_t gpj_result_num_queries(const gpj_result *r);
int64_t gpj_result_num_lines(const gpj_result *r);
int gpj_result_slots(const gpj_result *r);
/* Pointer to int64[num_queries][num_lines][slots][2], valid until release. */
const int64_t *gpj_result_offsets(const gpj_result *r);
/* The memory of the largest released result (up to 512 MiB) is kept for
 * the next result of the process: its pages are already mapped, which
 * makes that result's copy from the device several times cheaper. */
void gpj_result_release(gpj_result *r);

/* ---- values ------------------------------------------------------------------ */

/* Kinds of a (start, end) result pair in value extraction. */
#define GPJ_VALUE_NULL 0       /* start == -1: no match (ResultItem returns null) */
#define GPJ_VALUE_PRESENT 1    /* the bytes file[start, end) */
#define GPJ_VALUE_UNREADABLE 2 /* end before start (or past the file): the reference's
                                  ResultItem fails to build it (NegativeArraySizeException) */

/* Value extraction on the device (result/ResultItem.java:32-52 slices the
 * memory-mapped file on the host, one String per access): for `npairs`
 * (start, end) pairs of `file` in device memory (e.g. gpj_query_device
 * output), writes the kind of each pair to d_kinds[npairs], the byte offset
 * of its value to d_offsets[npairs + 1] (d_offsets[npairs] = the total;
 * non-values take no bytes) and the values back to back to d_bytes.  Returns
 * GPJ_ELIMIT with *total_bytes set when bytes_cap is too small (kinds and
 * offsets are complete then).  Synchronous. */
int gpj_values_device(gpj_ctx *ctx, gpj_file *file, const int64_t *d_pairs, int64_t npairs,
                      uint8_t *d_kinds, int64_t *d_offsets, uint8_t *d_bytes, int64_t bytes_cap,
                      int64_t *total_bytes);

/* gpj_query_paths with the values instead of the offsets: the paths are
 * evaluated as there, the values gathered on the device and copied to the
 * host compactly.  Item i = (query * lines + line) * slots + slot. */
int gpj_query_values(gpj_ctx *ctx, gpj_file *file, int nq, const char *const *paths,
                     gpj_values **out);
int64_t gpj_values_num_queries(const gpj_values *v);
int64_t gpj_values_num_lines(const gpj_values *v);
int gpj_values_slots(const gpj_values *v);
const uint8_t *gpj_values_kinds(const gpj_values *v);   /* [items] GPJ_VALUE_* */
const int64_t *gpj_values_offsets(const gpj_values *v); /* [items + 1] */
const uint8_t *gpj_values_bytes(const gpj_values *v);   /* gpj_values_size bytes */
int64_t gpj_values_size(const gpj_values *v);
void gpj_values_release(gpj_values *v);

/* ---- batches ---------------------------------------------------------------- */

/* Many (file, paths) requests evaluated together, with no counterpart call in
 * the reference (which handles one query() per call): gpj_batch_run indexes
 * every file of the batch whose index is missing or too shallow in one
 * kernel launch over all their tiles (plus one newline pass), evaluates every
 * request's queries over every line of every file in one find_value launch,
 * and copies all results back with one copy.  Files already indexed deeply
 * enough keep their index (a resident corpus is indexed once).  Results of
 * each request equal gpj_query_paths on its file alone.  Files must be of the
 * batch's device and stay valid until gpj_batch_run returns. */
typedef struct gpj_batch gpj_batch;
int gpj_batch_create(gpj_ctx *ctx, gpj_batch **out);
/* Adds a request; *item receives its number.  Paths are compiled here
 * (GPJ_EPARSE / GPJ_EUNSUPPORTED as gpj_compile). */
int gpj_batch_add(gpj_batch *batch, gpj_file *file, int nq, const char *const *paths, int *item);
int gpj_batch_run(gpj_batch *batch);
/* Results of request `item` of the last run (gpj_result layout, its queries
 * in the order added; slots = the largest num_results among the queries of
 * the request's file in this batch). */
int gpj_batch_result(gpj_batch *batch, int item, gpj_result **out);
/* The same with `slots` result slots per line (0: as gpj_batch_result):
 * each line's first `slots` slots, which hold every result of the request's
 * own queries when slots >= their largest num_results (GPJ_EINVAL when
 * slots exceeds the batch's slots for that file). */
int gpj_batch_result_ex(gpj_batch *batch, int item, int slots, gpj_result **out);
int gpj_batch_size(const gpj_batch *batch);
/* Removes all requests (the batch can be filled and run again). */
void gpj_batch_clear(gpj_batch *batch);
void gpj_batch_release(gpj_batch *batch);

/* ---- serving ----------------------------------------------------------------- */

/* A request server: (corpus, paths) requests against corpora kept resident
 * in device memory with their structural indexes under a byte budget, with
 * no counterpart in the reference (whose query() reads, indexes and queries
 * the file on every call, QueryFunction.java:48-265; a server would call the
 * interop object of GPJSONLibrary.java:48-54 once per request).
 *  - `workers` serving threads, each with its own context and stream: a
 *    free worker takes every pending request whose corpus is resident (up to
 *    max_batch, in arrival order) and evaluates them as one batch
 *    (gpj_batch_run); requests arriving meanwhile are taken by the next free
 *    worker, so iterations overlap on the device (continuous batching).
 *  - one loader thread: a corpus is loaded (copy from page-locked host
 *    memory pipelined with its index build) when a request needs it and its
 *    resident bytes fit the budget; least recently used corpora that no
 *    pending or running request needs are evicted, their bytes counting
 *    against the budget until their memory is released.
 * Every function is thread-safe.  A request's result equals gpj_query_paths
 * on its corpus alone (gpj_result layout; slots = the largest num_results of
 * its own paths). */
typedef struct gpj_server gpj_server;
typedef struct gpj_server_config {
    int32_t device;
    int32_t num_levels;    /* every corpus is indexed with this many levels (1..16); deeper paths are refused */
    int64_t budget_bytes;  /* device bytes for resident corpora with their indexes */
    int32_t max_batch;     /* requests per iteration (>= 1) */
    int32_t workers;       /* serving threads, iterations on the device at once (1..8) */
} gpj_server_config;

int gpj_serve_create(const gpj_server_config *cfg, gpj_server **out);
/* Registers n bytes of NDJSON in host memory as a corpus (*corpus = its
 * number).  The memory must stay valid and unchanged until
 * gpj_serve_destroy; it is page-locked here (cudaHostRegister) unless it
 * already is.  Nothing is loaded before a request needs it.  GPJ_ELIMIT when
 * its resident bytes exceed the budget. */
int gpj_serve_add_corpus(gpj_server *s, const void *host, int64_t n, int *corpus);
/* Requests per iteration and iterations at once from now on (max_inflight
 * is capped at the server's workers; 1, 1 = one request at a time). */
int gpj_serve_set_batching(gpj_server *s, int max_batch, int max_inflight);
/* Queues a request and returns at once; *request receives its id.  Paths
 * are compiled here: GPJ_EPARSE / GPJ_EUNSUPPORTED as gpj_compile,
 * GPJ_ELIMIT for a path deeper than the server's num_levels. */
int gpj_serve_submit(gpj_server *s, int corpus, int nq, const char *const *paths, uint64_t *request);
/* Waits up to timeout_ms (0: do not wait, -1: no limit) for request
 * `request`.  When it has finished, hands over its result (*out, released
 * with gpj_result_release) with its submit and completion times (ns since
 * the server's creation, optional) and returns its status; GPJ_EAGAIN while
 * it is not finished (call again). */
int gpj_serve_poll(gpj_server *s, uint64_t request, int timeout_ms, gpj_result **out, int64_t *submit_ns,
                   int64_t *done_ns);
/* The server's clock (ns since creation), as used by gpj_serve_poll. */
int64_t gpj_serve_now_ns(const gpj_server *s);
/* Counters as JSON (served, batches, loads, evictions, resident corpora,
 * budget bytes in use); writes at most cap bytes including the NUL, *len
 * receives the full length. */
int gpj_serve_stats(gpj_server *s, char *json, size_t cap, size_t *len);
/* Stops the threads, releases the resident corpora and unregisters the host
 * memory; requests not handed back are dropped. */
void gpj_serve_destroy(gpj_server *s);

/* ---- diagnostics ---------------------------------------------------------- */

/* Phase timings of the context as JSON (the role of Timings.export,
 * debug/Timings.java:50-88, with CUDA-event device times).  Writes at most
 * cap bytes including the NUL; *len receives the full length. */
int gpj_get_timings(gpj_ctx *ctx, char *json, size_t cap, size_t *len);
void gpj_reset_timings(gpj_ctx *ctx);

/* Number of kernels this context has launched since creation. */
int64_t gpj_kernel_launches(const gpj_ctx *ctx);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* GPJSON_B200_H */
