/*
 * gpjson_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of GPJSON's sequential structural-index and JSONPath
 * interpreter path, used as the checker for the CUDA path.  Only the test
 * suite, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
 * arm may load this library; the product library never links it.
 *
 * Parity status: pinned.  The restatement follows
 *   gpjson/src/main/java/com/koenv/gpjson/sequential/Sequential.java
 * line by line, widened to 64-bit offsets, and is checked against the
 * reference's own known answers (QueryFunctionTest.java:86-198) and
 * fixture-derived stage expectations (StringIndexTest.java:109-175,
 * NewlineIndexTest.java:81-115, LeveledBitmapsIndexTest.java:94-164).
 *
 * Where the reference is undefined (Java exception, device assert or
 * out-of-bounds access) this oracle fixes one behaviour and the CUDA path
 * implements the same one; each such point is marked "[bounded]" in the
 * source.
 */
#ifndef GPJSON_ORACLE_H
#define GPJSON_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Sequential.java:14-34.  Writes [0]=0 and then every '\n' offset; returns
 * the number of entries (newlines + 1).  Only the first `cap` are stored. */
int64_t gpjo_newline_index(const uint8_t *file, int64_t n, int64_t *out, int64_t cap);

/* Sequential.java:36-64.  out has ceil(n/64) words. */
void gpjo_string_index(const uint8_t *file, int64_t n, uint64_t *out);

/* Sequential.java:66-128.  out has num_levels * ceil(n/64) words,
 * level-major.  Levels below 0 are never marked [bounded]. */
void gpjo_leveled_bitmaps(const uint8_t *file, int64_t n, const uint64_t *string_index,
                          int num_levels, uint64_t *out);

/* Sequential.java:130-344.  Runs one compiled query over every line.
 * out has num_lines * 2 * result_size entries and is filled with -1 first. */
void gpjo_find_value(const uint8_t *file, int64_t n, const int64_t *newline_index,
                     int64_t num_lines, const uint64_t *string_index,
                     const uint64_t *leveled_bitmaps, int num_levels,
                     const uint8_t *ir, int64_t ir_len, int result_size, int64_t *out);

/* Multi-threaded variants used as the timed CPU baseline (same outputs). */
int64_t gpjo_newline_index_mt(const uint8_t *file, int64_t n, int64_t *out, int64_t cap);
void gpjo_string_index_mt(const uint8_t *file, int64_t n, uint64_t *out);
void gpjo_leveled_bitmaps_mt(const uint8_t *file, int64_t n, const uint64_t *string_index,
                             int num_levels, uint64_t *out);
void gpjo_find_value_mt(const uint8_t *file, int64_t n, const int64_t *newline_index,
                        int64_t num_lines, const uint64_t *string_index,
                        const uint64_t *leveled_bitmaps, int num_levels,
                        const uint8_t *ir, int64_t ir_len, int result_size, int64_t *out);

/* Number of OpenMP threads the *_mt variants use. */
int gpjo_num_threads(void);

#ifdef __cplusplus
}
#endif

#endif
