/*
 * gpjson_oracle.c — TEST INFRASTRUCTURE ONLY (see gpjson_oracle.h).
 *
 * A plain-C restatement of the reference's CPU path
 *   gpjson/src/main/java/com/koenv/gpjson/sequential/Sequential.java
 * with 64-bit offsets.  Every function cites the lines it follows.
 * The *_mt variants compute the same outputs with OpenMP over byte chunks
 * (index stages, carries resolved by a prefix over chunk summaries) or over
 * lines (interpreter); they exist to time the CPU baseline on all host cores.
 */
#include "gpjson_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum {
    OP_END = 0,          /* Opcode.java:4, ordinal 0 */
    OP_STORE_RESULT = 1, /* ordinal 1 */
    OP_MOVE_UP = 2,
    OP_MOVE_DOWN = 3,
    OP_MOVE_TO_KEY = 4,
    OP_MOVE_TO_INDEX = 5,
    OP_EXPRESSION_STRING_EQUALS = 6
};

/* The interpreter keeps one slot per level plus one, so that a query of the
 * maximum depth (16 key/index steps) can descend to level 16.  The reference
 * sizes these arrays at MAX_NUM_LEVELS=16 (Sequential.java:131,154,170). */
#define ORACLE_LEVEL_SLOTS 17

static inline int64_t words_for(int64_t n) { return (n + 63) / 64; }

static inline int bit_at(const uint64_t *bm, int64_t i) {
    return (int)((bm[i >> 6] >> (i & 63)) & 1u);
}

static inline int is_ws(uint8_t c) { return c == '\n' || c == '\r' || c == '\t' || c == ' '; }

/* ---------------------------------------------------------------------- */
/* Sequential.java:14-34                                                  */
int64_t gpjo_newline_index(const uint8_t *file, int64_t n, int64_t *out, int64_t cap) {
    int64_t count = 0;
    if (cap > 0) out[0] = 0; /* index.add(0L) (:19) */
    count = 1;
    for (int64_t i = 0; i < n; i++) {
        if (file[i] != '\n') continue;
        if (count < cap) out[count] = i; /* index.add(i) (:26) */
        count++;
    }
    return count;
}

/* Sequential.java:36-64                                                  */
void gpjo_string_index(const uint8_t *file, int64_t n, uint64_t *out) {
    memset(out, 0, (size_t)words_for(n) * 8);
    int escaped = 0;
    int in_string = 0;
    for (int64_t i = 0; i < n; i++) {
        if (file[i] == '"' && escaped != 1) in_string = !in_string; /* :44-46 */
        if (in_string) out[i / 64] |= (uint64_t)1 << (i % 64);     /* :48-50 */
        if (file[i] == '\\') escaped ^= 1;                          /* :52-56 */
        else escaped = 0;
    }
}

/* Sequential.java:66-128                                                 */
void gpjo_leveled_bitmaps(const uint8_t *file, int64_t n, const uint64_t *string_index,
                          int num_levels, uint64_t *out) {
    const int64_t level_size = words_for(n);
    memset(out, 0, (size_t)(level_size * num_levels) * 8);
    int64_t level = -1; /* :75 */
    for (int64_t i = 0; i < n; i++) {
        const uint64_t bit = (uint64_t)1 << (i % 64);
        if (string_index[i / 64] & bit) continue; /* :85 */
        const uint8_t v = file[i];
        if (v == '{' || v == '[') { /* :88-92 */
            level++;
            /* [bounded] the reference indexes a negative level here after an
             * unbalanced close (Java AIOOBE); negative levels are skipped. */
            if (level >= 0 && level < num_levels) out[level_size * level + i / 64] |= bit;
        } else if (v == '}' || v == ']') { /* :93-97 */
            if (level >= 0 && level < num_levels) out[level_size * level + i / 64] |= bit;
            level--;
        } else if ((v == ':' || v == ',') && level >= 0 && level < num_levels) { /* :98-101 */
            out[level_size * level + i / 64] |= bit;
        }
    }
}

/* ---------------------------------------------------------------------- */
/* IRByteInputBuffer.java:27-39 (LEB128, at most 5 bytes).                */
static int64_t read_varint(const uint8_t *ir, int64_t *pos) {
    int64_t value = 0;
    int shift = 0;
    int b;
    while (((b = ir[(*pos)++]) & 0x80) != 0) {
        value |= (int64_t)(b & 0x7F) << shift;
        shift += 7;
    }
    return value | ((int64_t)b << shift);
}

/* Sequential.java:130-344, one line.  `res` points at this line's
 * 2*result_size slots. */
static void find_value_line(const uint8_t *file, int64_t n, int64_t line_start, int64_t line_end,
                            const uint64_t *string_index, const uint64_t *lvl, int64_t level_size,
                            const uint8_t *ir, int64_t *res) {
    int64_t pc = 0;
    int cur = 0;
    int64_t level_ends[ORACLE_LEVEL_SLOTS];
    int64_t current_index[ORACLE_LEVEL_SLOTS];
    level_ends[0] = line_end; /* :155 */
    for (int k = 1; k < ORACLE_LEVEL_SLOTS; k++) level_ends[k] = -1;
    for (int k = 0; k < ORACLE_LEVEL_SLOTS; k++) current_index[k] = -1;
    int result_index = 0;
    int type = -1;
    int64_t looking_for_len = 0;
    const uint8_t *looking_for = 0;
    int64_t looking_for_index = -1;
    int execute = 1;

    for (int64_t j = line_start; j < level_ends[cur] && j < n; j++) { /* :179 */
        while (execute) {
            type = ir[pc++];
            switch (type) {
            case OP_END: /* :184-185 */
                return;
            case OP_STORE_RESULT: /* :186-207 */
                /* [bounded] the whitespace skip stops at the end of the file */
                while (j < n && is_ws(file[j])) j++;
                res[result_index * 2] = j;
                res[result_index * 2 + 1] = level_ends[cur];
                result_index++;
                break;
            case OP_MOVE_UP: /* :208-215 */
                /* [bounded] moving up out of a level whose end was never found
                 * would set j=-1 (the reference then reads file[-1]); the line
                 * ends instead. */
                if (level_ends[cur] < 0) return;
                j = level_ends[cur];
                level_ends[cur] = -1;
                cur--;
                break;
            case OP_MOVE_DOWN: /* :216-230 */
                cur++;
                if (level_ends[cur] == -1) {
                    for (int64_t m = j + 1; m < level_ends[cur - 1]; m++) {
                        if (bit_at(lvl + level_size * (cur - 1), m)) {
                            level_ends[cur] = m;
                            break;
                        }
                    }
                }
                break;
            case OP_MOVE_TO_KEY: /* :231-237 */
                looking_for_len = read_varint(ir, &pc);
                looking_for = ir + pc;
                pc += looking_for_len;
                execute = 0;
                break;
            case OP_MOVE_TO_INDEX: /* :238-266 */
                looking_for_index = read_varint(ir, &pc);
                if (current_index[cur] == -1) {
                    for (;;) {
                        /* [bounded] the reference asserts that only whitespace
                         * precedes '[' and that the file does not end; a line
                         * where that fails ends here. */
                        if (j >= n) return;
                        const uint8_t c = file[j];
                        if (c == '[') break;
                        if (!is_ws(c)) return;
                        j++;
                    }
                    current_index[cur] = 0;
                }
                if (looking_for_index == 0) {
                    j++;
                    execute = 1;
                } else {
                    execute = 0;
                }
                break;
            case OP_EXPRESSION_STRING_EQUALS: { /* :267-293 */
                looking_for_len = read_varint(ir, &pc);
                looking_for = ir + pc;
                pc += looking_for_len;
                while (j < n && is_ws(file[j])) j++; /* [bounded] */
                const int64_t actual = level_ends[cur] - j;
                if (actual != looking_for_len) return;
                for (int64_t k = 0; k < looking_for_len; k++)
                    if (looking_for[k] != file[j + k]) return;
                break;
            }
            default:
                return; /* unreachable for validated bytecode */
            }
        }

        /* [bounded] the reference also runs this check when an opcode above
         * moved j to the end of the file, reading past the buffer. */
        if (j >= n) continue;
        const int structural = bit_at(lvl + level_size * cur, j); /* :299 */
        if (type == OP_MOVE_TO_KEY) { /* :301-327 */
            if (structural && file[j] == ':') {
                int64_t string_end = -1;
                for (int64_t k = j - 1; k > line_start; k--) {
                    if (bit_at(string_index, k)) {
                        string_end = k;
                        break;
                    }
                }
                const int64_t string_start = string_end - looking_for_len;
                if (string_start < line_start || file[string_start] != '"') continue;
                execute = 1;
                for (int64_t k = 0; k < looking_for_len; k++) {
                    if (looking_for[k] != file[string_start + k + 1]) {
                        execute = 0;
                        break;
                    }
                }
            }
        } else if (type == OP_MOVE_TO_INDEX) { /* :328-335 */
            if (structural && file[j] == ',') {
                current_index[cur]++;
                if (looking_for_index == current_index[cur]) execute = 1;
            }
        }
    }
}

void gpjo_find_value(const uint8_t *file, int64_t n, const int64_t *newline_index,
                     int64_t num_lines, const uint64_t *string_index,
                     const uint64_t *leveled_bitmaps, int num_levels,
                     const uint8_t *ir, int64_t ir_len, int result_size, int64_t *out) {
    (void)ir_len;
    (void)num_levels;
    const int64_t level_size = words_for(n);
    const int64_t total = num_lines * 2 * (int64_t)result_size;
    for (int64_t k = 0; k < total; k++) out[k] = -1; /* :143-144 */
    for (int64_t i = 0; i < num_lines; i++) {       /* :146 */
        const int64_t start = newline_index[i];
        const int64_t end = (i + 1 < num_lines) ? newline_index[i + 1] : n; /* :148 */
        find_value_line(file, n, start, end, string_index, leveled_bitmaps, level_size, ir,
                        out + i * 2 * (int64_t)result_size);
    }
}

/* ---------------------------------------------------------------------- */
/* Multi-threaded variants (CPU baseline).                                */

int gpjo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Chunk boundaries on multiples of 64 bytes so that no two threads write
 * the same bitmap word. */
static int64_t chunk_bytes_for(int64_t n, int nthreads) {
    int64_t c = (n + nthreads * 4 - 1) / (nthreads * 4);
    c = (c + 63) & ~(int64_t)63;
    if (c < 4096) c = 4096;
    return c;
}

int64_t gpjo_newline_index_mt(const uint8_t *file, int64_t n, int64_t *out, int64_t cap) {
    const int nt = gpjo_num_threads();
    const int64_t cb = chunk_bytes_for(n, nt);
    const int64_t nchunks = (n + cb - 1) / cb;
    int64_t *counts = (int64_t *)calloc((size_t)nchunks + 1, sizeof(int64_t));
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nchunks; c++) {
        const int64_t s = c * cb, e = (s + cb < n) ? s + cb : n;
        int64_t k = 0;
        for (int64_t i = s; i < e; i++) k += file[i] == '\n';
        counts[c + 1] = k;
    }
    counts[0] = 1;
    for (int64_t c = 1; c <= nchunks; c++) counts[c] += counts[c - 1];
    if (cap > 0) out[0] = 0;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nchunks; c++) {
        const int64_t s = c * cb, e = (s + cb < n) ? s + cb : n;
        int64_t k = counts[c];
        for (int64_t i = s; i < e; i++)
            if (file[i] == '\n') {
                if (k < cap) out[k] = i;
                k++;
            }
    }
    const int64_t total = counts[nchunks];
    free(counts);
    return total;
}

/* Escape state at byte `pos`: parity of the backslash run ending at pos-1. */
static int escape_state_before(const uint8_t *file, int64_t pos) {
    int64_t k = pos - 1, run = 0;
    while (k >= 0 && file[k] == '\\') {
        run++;
        k--;
    }
    return (int)(run & 1);
}

void gpjo_string_index_mt(const uint8_t *file, int64_t n, uint64_t *out) {
    const int nt = gpjo_num_threads();
    const int64_t cb = chunk_bytes_for(n, nt);
    const int64_t nchunks = (n + cb - 1) / cb;
    uint8_t *parity = (uint8_t *)calloc((size_t)nchunks + 1, 1);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nchunks; c++) {
        const int64_t s = c * cb, e = (s + cb < n) ? s + cb : n;
        int escaped = escape_state_before(file, s);
        int q = 0;
        for (int64_t i = s; i < e; i++) {
            if (file[i] == '"' && escaped != 1) q ^= 1;
            if (file[i] == '\\') escaped ^= 1;
            else escaped = 0;
        }
        parity[c + 1] = (uint8_t)q;
    }
    for (int64_t c = 1; c <= nchunks; c++) parity[c] ^= parity[c - 1];
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nchunks; c++) {
        const int64_t s = c * cb, e = (s + cb < n) ? s + cb : n;
        int escaped = escape_state_before(file, s);
        int in_string = parity[c];
        for (int64_t w = s / 64; w < (e + 63) / 64; w++) out[w] = 0;
        for (int64_t i = s; i < e; i++) {
            if (file[i] == '"' && escaped != 1) in_string = !in_string;
            if (in_string) out[i / 64] |= (uint64_t)1 << (i % 64);
            if (file[i] == '\\') escaped ^= 1;
            else escaped = 0;
        }
    }
    free(parity);
}

void gpjo_leveled_bitmaps_mt(const uint8_t *file, int64_t n, const uint64_t *string_index,
                             int num_levels, uint64_t *out) {
    const int nt = gpjo_num_threads();
    const int64_t cb = chunk_bytes_for(n, nt);
    const int64_t nchunks = (n + cb - 1) / cb;
    const int64_t level_size = words_for(n);
    int64_t *depth = (int64_t *)calloc((size_t)nchunks + 1, sizeof(int64_t));
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nchunks; c++) {
        const int64_t s = c * cb, e = (s + cb < n) ? s + cb : n;
        int64_t d = 0;
        for (int64_t i = s; i < e; i++) {
            if (bit_at(string_index, i)) continue;
            const uint8_t v = file[i];
            d += (v == '{' || v == '[') - (v == '}' || v == ']');
        }
        depth[c + 1] = d;
    }
    depth[0] = -1;
    for (int64_t c = 1; c <= nchunks; c++) depth[c] += depth[c - 1];
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nchunks; c++) {
        const int64_t s = c * cb, e = (s + cb < n) ? s + cb : n;
        for (int l = 0; l < num_levels; l++)
            for (int64_t w = s / 64; w < (e + 63) / 64; w++) out[level_size * l + w] = 0;
        int64_t level = depth[c];
        for (int64_t i = s; i < e; i++) {
            const uint64_t bit = (uint64_t)1 << (i % 64);
            if (string_index[i / 64] & bit) continue;
            const uint8_t v = file[i];
            if (v == '{' || v == '[') {
                level++;
                if (level >= 0 && level < num_levels) out[level_size * level + i / 64] |= bit;
            } else if (v == '}' || v == ']') {
                if (level >= 0 && level < num_levels) out[level_size * level + i / 64] |= bit;
                level--;
            } else if ((v == ':' || v == ',') && level >= 0 && level < num_levels) {
                out[level_size * level + i / 64] |= bit;
            }
        }
    }
    free(depth);
}

void gpjo_find_value_mt(const uint8_t *file, int64_t n, const int64_t *newline_index,
                        int64_t num_lines, const uint64_t *string_index,
                        const uint64_t *leveled_bitmaps, int num_levels,
                        const uint8_t *ir, int64_t ir_len, int result_size, int64_t *out) {
    (void)ir_len;
    (void)num_levels;
    const int64_t level_size = words_for(n);
    const int64_t r2 = 2 * (int64_t)result_size;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < num_lines; i++) {
        int64_t *res = out + i * r2;
        for (int64_t k = 0; k < r2; k++) res[k] = -1;
        const int64_t start = newline_index[i];
        const int64_t end = (i + 1 < num_lines) ? newline_index[i + 1] : n;
        find_value_line(file, n, start, end, string_index, leveled_bitmaps, level_size, ir, res);
    }
}
