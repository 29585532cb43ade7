package com.koenv.gpjson.gpu;

import com.koenv.gpjson.GPJSONException;
import java.lang.foreign.Arena;
import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.Linker;
import java.lang.foreign.MemoryLayout;
import java.lang.foreign.MemorySegment;
import java.lang.foreign.SymbolLookup;
import java.lang.invoke.MethodHandle;
import java.nio.file.Path;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_INT;
import static java.lang.foreign.ValueLayout.JAVA_LONG;

/**
 * Panama FFM (Java 22+) binding of libgpjson_b200 (include/gpjson_b200.h),
 * the drop-in for the grCUDA-derived runtime GPJSON's query path runs on
 * (gpu/CUDARuntime.java:76-94, its NFI bindings gpu/CUDARuntimeFunction.java:39-186
 * and the NVRTC compiler gpu/NVRuntimeCompiler.java): QueryFunction.call keeps
 * its argument checks and calls {@link #query}; the offsets it returns
 * (long[query][line][slot][2], -1 = miss) feed Result / ResultArray /
 * ResultItem unchanged.  One handle per C entry point; every descriptor
 * follows the declaration in the header (int / unsigned / int32_t:
 * JAVA_INT, int64_t / uint64_t / size_t: JAVA_LONG, pointers: ADDRESS).
 * The library path comes from the system property gpjson.b200.lib.
 */
public final class GpjNative implements AutoCloseable {
    private static final Linker LINKER = Linker.nativeLinker();
    private static final SymbolLookup LIB =
            SymbolLookup.libraryLookup(System.getProperty("gpjson.b200.lib", "libgpjson_b200.so"), Arena.global());

    private static MethodHandle fn(String name, FunctionDescriptor d) {
        return LINKER.downcallHandle(LIB.find(name).orElseThrow(), d);
    }

    // ---- context
    static final MethodHandle CREATE = fn("gpj_create", FunctionDescriptor.of(JAVA_INT, JAVA_INT, ADDRESS));
    static final MethodHandle DESTROY = fn("gpj_destroy", FunctionDescriptor.ofVoid(ADDRESS));
    static final MethodHandle LAST_ERROR = fn("gpj_last_error", FunctionDescriptor.of(ADDRESS, ADDRESS));
    static final MethodHandle SET_STREAM = fn("gpj_set_stream", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
    static final MethodHandle SET_TUNING = fn("gpj_set_tuning", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
    static final MethodHandle GET_TUNING = fn("gpj_get_tuning", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
    static final MethodHandle SET_QUERY_FUSION =
            fn("gpj_set_query_fusion", FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT));
    static final MethodHandle SET_PATH_EXTENSIONS =
            fn("gpj_set_path_extensions", FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT));
    static final MethodHandle VERSION = fn("gpj_version", FunctionDescriptor.of(ADDRESS));

    // ---- JSONPath compiler (byte-identical to JSONPathParser.compile)
    static final MethodHandle COMPILE = fn("gpj_compile", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG,
            ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_LONG));
    static final MethodHandle COMPILE_EX = fn("gpj_compile_ex", FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT,
            ADDRESS, JAVA_LONG, ADDRESS, ADDRESS, ADDRESS, ADDRESS, JAVA_LONG));

    // ---- files (readFile, QueryFunction.java:316-335)
    static final MethodHandle FILE_OPEN =
            fn("gpj_file_open", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS));
    static final MethodHandle FILE_FROM_HOST =
            fn("gpj_file_from_host", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG, ADDRESS));
    static final MethodHandle FILE_FROM_HOST_INDEXED = fn("gpj_file_from_host_indexed",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG, JAVA_INT, ADDRESS));
    static final MethodHandle FILE_FROM_HOST_QUERY = fn("gpj_file_from_host_query",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG, JAVA_INT, JAVA_INT, ADDRESS, ADDRESS,
                    JAVA_INT, ADDRESS, JAVA_LONG, ADDRESS, ADDRESS));
    static final MethodHandle FILE_FROM_DEVICE =
            fn("gpj_file_from_device", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG, ADDRESS));
    static final MethodHandle FILE_RELEASE = fn("gpj_file_release", FunctionDescriptor.ofVoid(ADDRESS));
    static final MethodHandle FILE_SIZE = fn("gpj_file_size", FunctionDescriptor.of(JAVA_LONG, ADDRESS));

    // ---- index (CombinedIndex + LeveledBitmapsIndex)
    static final MethodHandle INDEX_BUILD =
            fn("gpj_index_build", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT));
    static final MethodHandle INDEX_NUM_LINES =
            fn("gpj_index_num_lines", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
    static final MethodHandle INDEX_COPY_NEWLINES = fn("gpj_index_copy_newlines",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_LONG));
    static final MethodHandle INDEX_COPY_STRING_INDEX = fn("gpj_index_copy_string_index",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_LONG));
    static final MethodHandle INDEX_COPY_LEVELED_BITMAPS = fn("gpj_index_copy_leveled_bitmaps",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_LONG));
    static final MethodHandle BUILD_INDEX_DEVICE = fn("gpj_build_index_device", FunctionDescriptor.of(JAVA_INT,
            ADDRESS, ADDRESS, JAVA_LONG, JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_LONG, ADDRESS));
    static final MethodHandle BUILD_INDEX_DEVICE_NOALLOC = fn("gpj_build_index_device_noalloc",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG, JAVA_INT, ADDRESS, ADDRESS, ADDRESS,
                    JAVA_LONG, ADDRESS));

    // ---- queries (the per-query find_value launches, QueryFunction.java:194-241)
    static final MethodHandle QUERY = fn("gpj_query", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT,
            ADDRESS, ADDRESS, JAVA_INT, ADDRESS, JAVA_LONG));
    static final MethodHandle QUERY_DEVICE = fn("gpj_query_device", FunctionDescriptor.of(JAVA_INT, ADDRESS,
            ADDRESS, JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, JAVA_LONG));
    static final MethodHandle INDEX_QUERY_DEVICE = fn("gpj_index_query_device", FunctionDescriptor.of(JAVA_INT,
            ADDRESS, ADDRESS, JAVA_INT, JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, JAVA_LONG));
    static final MethodHandle QUERY_PATHS = fn("gpj_query_paths",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS));

    // ---- results (Result / ResultArray / ResultItem layout)
    static final MethodHandle RESULT_NUM_QUERIES =
            fn("gpj_result_num_queries", FunctionDescriptor.of(JAVA_LONG, ADDRESS));
    static final MethodHandle RESULT_NUM_LINES = fn("gpj_result_num_lines", FunctionDescriptor.of(JAVA_LONG, ADDRESS));
    static final MethodHandle RESULT_SLOTS = fn("gpj_result_slots", FunctionDescriptor.of(JAVA_INT, ADDRESS));
    static final MethodHandle RESULT_OFFSETS = fn("gpj_result_offsets", FunctionDescriptor.of(ADDRESS, ADDRESS));
    static final MethodHandle RESULT_RELEASE = fn("gpj_result_release", FunctionDescriptor.ofVoid(ADDRESS));

    // ---- values gathered on the device (ResultItem.readArrayElement, ResultItem.java:32-52)
    static final MethodHandle VALUES_DEVICE = fn("gpj_values_device", FunctionDescriptor.of(JAVA_INT, ADDRESS,
            ADDRESS, ADDRESS, JAVA_LONG, ADDRESS, ADDRESS, ADDRESS, JAVA_LONG, ADDRESS));
    static final MethodHandle QUERY_VALUES = fn("gpj_query_values",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS));
    static final MethodHandle VALUES_NUM_QUERIES =
            fn("gpj_values_num_queries", FunctionDescriptor.of(JAVA_LONG, ADDRESS));
    static final MethodHandle VALUES_NUM_LINES = fn("gpj_values_num_lines", FunctionDescriptor.of(JAVA_LONG, ADDRESS));
    static final MethodHandle VALUES_SLOTS = fn("gpj_values_slots", FunctionDescriptor.of(JAVA_INT, ADDRESS));
    static final MethodHandle VALUES_KINDS = fn("gpj_values_kinds", FunctionDescriptor.of(ADDRESS, ADDRESS));
    static final MethodHandle VALUES_OFFSETS = fn("gpj_values_offsets", FunctionDescriptor.of(ADDRESS, ADDRESS));
    static final MethodHandle VALUES_BYTES = fn("gpj_values_bytes", FunctionDescriptor.of(ADDRESS, ADDRESS));
    static final MethodHandle VALUES_SIZE = fn("gpj_values_size", FunctionDescriptor.of(JAVA_LONG, ADDRESS));
    static final MethodHandle VALUES_RELEASE = fn("gpj_values_release", FunctionDescriptor.ofVoid(ADDRESS));

    // ---- batches
    static final MethodHandle BATCH_CREATE = fn("gpj_batch_create", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
    static final MethodHandle BATCH_ADD = fn("gpj_batch_add",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT, ADDRESS, ADDRESS));
    static final MethodHandle BATCH_RUN = fn("gpj_batch_run", FunctionDescriptor.of(JAVA_INT, ADDRESS));
    static final MethodHandle BATCH_RESULT =
            fn("gpj_batch_result", FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS));
    static final MethodHandle BATCH_RESULT_EX =
            fn("gpj_batch_result_ex", FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, JAVA_INT, ADDRESS));
    static final MethodHandle BATCH_SIZE = fn("gpj_batch_size", FunctionDescriptor.of(JAVA_INT, ADDRESS));
    static final MethodHandle BATCH_CLEAR = fn("gpj_batch_clear", FunctionDescriptor.ofVoid(ADDRESS));
    static final MethodHandle BATCH_RELEASE = fn("gpj_batch_release", FunctionDescriptor.ofVoid(ADDRESS));

    // ---- request server (resident corpora, continuous batching)
    static final MethodHandle SERVE_CREATE = fn("gpj_serve_create", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
    static final MethodHandle SERVE_ADD_CORPUS = fn("gpj_serve_add_corpus",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG, ADDRESS));
    static final MethodHandle SERVE_SET_BATCHING =
            fn("gpj_serve_set_batching", FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, JAVA_INT));
    static final MethodHandle SERVE_SUBMIT = fn("gpj_serve_submit",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, JAVA_INT, ADDRESS, ADDRESS));
    static final MethodHandle SERVE_POLL = fn("gpj_serve_poll",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_LONG, JAVA_INT, ADDRESS, ADDRESS, ADDRESS));
    static final MethodHandle SERVE_NOW_NS = fn("gpj_serve_now_ns", FunctionDescriptor.of(JAVA_LONG, ADDRESS));
    static final MethodHandle SERVE_STATS =
            fn("gpj_serve_stats", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG, ADDRESS));
    static final MethodHandle SERVE_DESTROY = fn("gpj_serve_destroy", FunctionDescriptor.ofVoid(ADDRESS));

    // ---- diagnostics (Timings.export, debug/Timings.java:50-88)
    static final MethodHandle GET_TIMINGS =
            fn("gpj_get_timings", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG, ADDRESS));
    static final MethodHandle RESET_TIMINGS = fn("gpj_reset_timings", FunctionDescriptor.ofVoid(ADDRESS));
    static final MethodHandle KERNEL_LAUNCHES = fn("gpj_kernel_launches", FunctionDescriptor.of(JAVA_LONG, ADDRESS));

    /** gpj_server_config (device, num_levels, budget_bytes, max_batch, workers). */
    public static final MemoryLayout SERVER_CONFIG = MemoryLayout.structLayout(JAVA_INT.withName("device"),
            JAVA_INT.withName("num_levels"), JAVA_LONG.withName("budget_bytes"), JAVA_INT.withName("max_batch"),
            JAVA_INT.withName("workers"));

    static final int GPJ_OK = 0, GPJ_EPARSE = -2, GPJ_EUNSUPPORTED = -3, GPJ_EAGAIN = -10;

    private final MemorySegment ctx;

    public GpjNative(int device) throws Throwable {
        try (Arena a = Arena.ofConfined()) {
            MemorySegment out = a.allocate(ADDRESS);
            check((int) CREATE.invokeExact(device, out), MemorySegment.NULL);
            ctx = out.get(ADDRESS, 0);
        }
    }

    /** query(file, paths) of QueryFunction.call: offsets[q][line][slot][2] as one long[]; shapeOut = {nq, lines, slots}. */
    public long[] query(Path file, String[] paths, long[] shapeOut) throws Throwable {
        try (Arena a = Arena.ofConfined()) {
            MemorySegment fileOut = a.allocate(ADDRESS);
            check((int) FILE_OPEN.invokeExact(ctx, a.allocateFrom(file.toString()), fileOut), ctx);
            MemorySegment f = fileOut.get(ADDRESS, 0);
            try {
                MemorySegment arr = a.allocate(ADDRESS, paths.length);
                for (int i = 0; i < paths.length; i++) arr.setAtIndex(ADDRESS, i, a.allocateFrom(paths[i]));
                MemorySegment resOut = a.allocate(ADDRESS);
                check((int) QUERY_PATHS.invokeExact(ctx, f, paths.length, arr, resOut), ctx);
                return takeResult(resOut.get(ADDRESS, 0), shapeOut);
            } finally {
                FILE_RELEASE.invokeExact(f);
            }
        }
    }

    /** Copies a gpj_result out (and releases it); shapeOut = {nq, lines, slots}. */
    static long[] takeResult(MemorySegment r, long[] shapeOut) throws Throwable {
        try {
            long nq = (long) RESULT_NUM_QUERIES.invokeExact(r), lines = (long) RESULT_NUM_LINES.invokeExact(r);
            int slots = (int) RESULT_SLOTS.invokeExact(r);
            MemorySegment off = ((MemorySegment) RESULT_OFFSETS.invokeExact(r)).reinterpret(nq * lines * slots * 2 * 8);
            shapeOut[0] = nq;
            shapeOut[1] = lines;
            shapeOut[2] = slots;
            return off.toArray(JAVA_LONG);
        } finally {
            RESULT_RELEASE.invokeExact(r);
        }
    }

    static void check(int rc, MemorySegment ctx) throws Throwable {
        if (rc == GPJ_OK) return;
        String msg = ((MemorySegment) LAST_ERROR.invokeExact(ctx)).reinterpret(4096).getString(0);
        // GPJ_EPARSE / GPJ_EUNSUPPORTED are JSONPathException /
        // UnsupportedJSONPathException in QueryFunction, which may then fall back
        throw new GPJSONException(rc, msg, new String[] {"gpjson_b200"});
    }

    @Override
    public void close() throws Throwable {
        DESTROY.invokeExact(ctx);
    }

    /**
     * The request server for a host that serves many (corpus, paths)
     * requests: corpora registered once stay resident under a device byte
     * budget; requests from any thread are batched continuously.
     */
    public static final class Server implements AutoCloseable {
        private final MemorySegment s;

        public Server(int device, int numLevels, long budgetBytes, int maxBatch, int workers) throws Throwable {
            try (Arena a = Arena.ofConfined()) {
                MemorySegment cfg = a.allocate(SERVER_CONFIG);
                cfg.set(JAVA_INT, 0, device);
                cfg.set(JAVA_INT, 4, numLevels);
                cfg.set(JAVA_LONG, 8, budgetBytes);
                cfg.set(JAVA_INT, 16, maxBatch);
                cfg.set(JAVA_INT, 20, workers);
                MemorySegment out = a.allocate(ADDRESS);
                check((int) SERVE_CREATE.invokeExact(cfg, out), MemorySegment.NULL);
                s = out.get(ADDRESS, 0);
            }
        }

        /** Registers a corpus; `data` (e.g. a mapped file) must outlive the server. */
        public int addCorpus(MemorySegment data) throws Throwable {
            try (Arena a = Arena.ofConfined()) {
                MemorySegment id = a.allocate(JAVA_INT);
                check((int) SERVE_ADD_CORPUS.invokeExact(s, data, data.byteSize(), id), MemorySegment.NULL);
                return id.get(JAVA_INT, 0);
            }
        }

        public long submit(int corpus, String[] paths) throws Throwable {
            try (Arena a = Arena.ofConfined()) {
                MemorySegment arr = a.allocate(ADDRESS, paths.length);
                for (int i = 0; i < paths.length; i++) arr.setAtIndex(ADDRESS, i, a.allocateFrom(paths[i]));
                MemorySegment id = a.allocate(JAVA_LONG);
                check((int) SERVE_SUBMIT.invokeExact(s, corpus, paths.length, arr, id), MemorySegment.NULL);
                return id.get(JAVA_LONG, 0);
            }
        }

        /** Waits for a request (timeoutMs -1: no limit); null while it is not finished. */
        public long[] poll(long request, int timeoutMs, long[] shapeOut) throws Throwable {
            try (Arena a = Arena.ofConfined()) {
                MemorySegment out = a.allocate(ADDRESS);
                int rc = (int) SERVE_POLL.invokeExact(s, request, timeoutMs, out, MemorySegment.NULL,
                        MemorySegment.NULL);
                if (rc == GPJ_EAGAIN) return null;
                MemorySegment r = out.get(ADDRESS, 0);
                if (rc != GPJ_OK) {
                    if (!r.equals(MemorySegment.NULL)) RESULT_RELEASE.invokeExact(r);
                    check(rc, MemorySegment.NULL);
                }
                return takeResult(r, shapeOut);
            }
        }

        @Override
        public void close() throws Throwable {
            SERVE_DESTROY.invokeExact(s);
        }
    }
}
