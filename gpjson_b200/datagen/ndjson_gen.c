/*
 * Seeded synthetic NDJSON of the benchmark shapes (the reference's Pison /
 * Twitter datasets are not available; datasets/README.md:3-18).
 *
 *  - gpjgen_tweets: tweet-like objects, ~1.5 KB mean per line: id int64,
 *    text of 20-280 chars (lognormal) with 5% multibyte and 1% escapes
 *    (\" \\ \n é), user {id, name, lang from 20 codes, followers_count
 *    log-uniform 0-1e7, ...}, entities {hashtags: 0-5 {text}} with a given
 *    share of empty arrays; nesting depth 4.
 *  - gpjgen_adversarial: line lengths log-uniform 100 B - 1 MiB, filler
 *    nesting depth uniform 1-16, arrays of 0-1000 ints/floats, strings
 *    where 10% carry backslash runs of length 1-7 (valid JSON escapes,
 *    including \\\"), and the fields a.b.c.d, arr[5], x[0].y[2].z present
 *    with 10-50% misses (index steps only ever meet arrays).
 *
 * Output is LF-terminated lines.  The buffer is filled in independent
 * blocks, each from its own seed, so the bytes do not depend on the thread
 * count.  Returns the number of bytes written (<= cap).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define GPJGEN_API __attribute__((visibility("default")))

typedef struct {
    uint64_t s;
} rng_t;

static inline uint64_t next64(rng_t *r) { /* splitmix64 */
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline double unif(rng_t *r) { return (double)(next64(r) >> 11) * (1.0 / 9007199254740992.0); }
static inline int64_t irange(rng_t *r, int64_t lo, int64_t hi) { /* inclusive */
    return lo + (int64_t)(next64(r) % (uint64_t)(hi - lo + 1));
}
static double normal(rng_t *r) {
    double u1 = unif(r), u2 = unif(r);
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

typedef struct {
    uint8_t *p, *end;
    int full;
} buf_t;

static inline void put(buf_t *b, const char *s, size_t n) {
    if (b->full || (size_t)(b->end - b->p) < n) {
        b->full = 1;
        return;
    }
    memcpy(b->p, s, n);
    b->p += n;
}
static inline void puts_(buf_t *b, const char *s) { put(b, s, strlen(s)); }
static inline void putc_(buf_t *b, char c) { put(b, &c, 1); }
static void put_int(buf_t *b, int64_t v) {
    char tmp[24];
    int n = 0, neg = v < 0;
    uint64_t u = neg ? (uint64_t)(-v) : (uint64_t)v;
    do {
        tmp[n++] = (char)('0' + u % 10);
        u /= 10;
    } while (u);
    if (neg) tmp[n++] = '-';
    char out[24];
    for (int i = 0; i < n; i++) out[i] = tmp[n - 1 - i];
    put(b, out, (size_t)n);
}

static const char *kWords[] = {"the", "gpu", "json", "data", "query", "fast", "index", "line",
                               "value", "string", "path", "level", "bitmap", "scan", "warp", "tile",
                               "hello", "world", "today", "great", "news", "love", "time", "new"};
#define NWORDS (sizeof(kWords) / sizeof(kWords[0]))
static const char *kLangs[20] = {"en", "nl", "de", "fr", "es", "it", "pt", "ja", "ko", "zh",
                                 "ru", "ar", "tr", "pl", "sv", "fi", "da", "no", "id", "th"};

/* Body of a JSON string of about `len` bytes (without quotes). */
static void put_text(buf_t *b, rng_t *r, int len, int multibyte, int escapes) {
    int w = 0;
    while (w < len && !b->full) {
        if (w) {
            putc_(b, ' ');
            w++;
        }
        const char *word = kWords[next64(r) % NWORDS];
        puts_(b, word);
        w += (int)strlen(word);
        if (multibyte && unif(r) < 0.15) {
            puts_(b, "\xc3\xa9");
            w += 2;
        }
        if (escapes && unif(r) < 0.2) {
            switch (next64(r) % 4) {
                case 0: puts_(b, "\\\""); break;
                case 1: puts_(b, "\\\\"); break;
                case 2: puts_(b, "\\n"); break;
                default: puts_(b, "\\u00e9"); break;
            }
            w += 2;
        }
    }
}

static void put_quoted_words(buf_t *b, rng_t *r, int len) {
    putc_(b, '"');
    put_text(b, r, len, 0, 0);
    putc_(b, '"');
}

/* One tweet-like line (without the trailing newline). */
static void tweet(buf_t *b, rng_t *r, int64_t id, double p_empty) {
    int text_len = (int)exp(log(80.0) + 0.6 * normal(r));
    if (text_len < 20) text_len = 20;
    if (text_len > 280) text_len = 280;
    const int multibyte = unif(r) < 0.05, escapes = unif(r) < 0.01;
    puts_(b, "{\"created_at\":\"Mon Apr 26 ");
    put_int(b, irange(r, 10, 23));
    puts_(b, ":");
    put_int(b, irange(r, 10, 59));
    puts_(b, ":00 +0000 2021\",\"id\":");
    put_int(b, id);
    puts_(b, ",\"id_str\":\"");
    put_int(b, id);
    puts_(b, "\",\"text\":\"");
    put_text(b, r, text_len, multibyte, escapes);
    puts_(b, "\",\"source\":\"<a href=\\\"https://example.com/app\\\" rel=\\\"nofollow\\\">App</a>\","
             "\"truncated\":false,\"in_reply_to_status_id\":null,\"in_reply_to_user_id\":null,"
             "\"user\":{\"id\":");
    put_int(b, (int64_t)(next64(r) >> 12));
    puts_(b, ",\"name\":");
    put_quoted_words(b, r, (int)irange(r, 5, 20));
    puts_(b, ",\"screen_name\":");
    put_quoted_words(b, r, (int)irange(r, 5, 15));
    puts_(b, ",\"location\":");
    put_quoted_words(b, r, (int)irange(r, 0, 30));
    puts_(b, ",\"description\":");
    put_quoted_words(b, r, (int)irange(r, 0, 160));
    puts_(b, ",\"url\":null,\"protected\":false,\"followers_count\":");
    put_int(b, (int64_t)floor(exp(unif(r) * log(1e7 + 1.0)) - 1.0));
    puts_(b, ",\"friends_count\":");
    put_int(b, irange(r, 0, 5000));
    puts_(b, ",\"listed_count\":");
    put_int(b, irange(r, 0, 100));
    puts_(b, ",\"favourites_count\":");
    put_int(b, irange(r, 0, 100000));
    puts_(b, ",\"statuses_count\":");
    put_int(b, irange(r, 0, 100000));
    puts_(b, ",\"verified\":false,\"profile_background_color\":\"C0DEED\",\"profile_link_color\":\"1DA1F2\","
             "\"profile_sidebar_border_color\":\"C0DEED\",\"profile_text_color\":\"333333\","
             "\"profile_use_background_image\":true,\"profile_banner_url\":\"https://example.com/banners/");
    put_int(b, irange(r, 100000, 999999));
    puts_(b, "/1600000000\",\"time_zone\":null,\"utc_offset\":null,\"geo_enabled\":false,"
             "\"contributors_enabled\":false,\"is_translator\":false,\"following\":null,"
             "\"follow_request_sent\":null,\"notifications\":null,\"lang\":\"");
    puts_(b, kLangs[next64(r) % 20]);
    puts_(b, "\",\"profile_image_url\":\"https://example.com/img/");
    put_int(b, irange(r, 100000, 999999));
    puts_(b, "_normal.jpg\",\"default_profile\":true},\"geo\":null,\"coordinates\":null,\"place\":null,"
             "\"contributors\":null,\"is_quote_status\":false,\"quote_count\":0,\"reply_count\":0,\"retweet_count\":");
    put_int(b, irange(r, 0, 1000));
    puts_(b, ",\"favorite_count\":");
    put_int(b, irange(r, 0, 1000));
    puts_(b, ",\"entities\":{\"hashtags\":[");
    const int nh = unif(r) < p_empty ? 0 : (int)irange(r, 1, 5);
    for (int h = 0; h < nh; h++) {
        if (h) putc_(b, ',');
        puts_(b, "{\"text\":");
        put_quoted_words(b, r, (int)irange(r, 3, 15));
        puts_(b, ",\"indices\":[");
        put_int(b, irange(r, 0, 100));
        putc_(b, ',');
        put_int(b, irange(r, 100, 140));
        puts_(b, "]}");
    }
    puts_(b, "],\"urls\":[],\"user_mentions\":[],\"symbols\":[]},\"favorited\":false,\"retweeted\":false,"
             "\"filter_level\":\"low\",\"lang\":\"");
    puts_(b, kLangs[next64(r) % 20]);
    puts_(b, "\",\"timestamp_ms\":\"16194");
    put_int(b, irange(r, 10000000, 99999999));
    puts_(b, "\"}");
}

/* A string whose body has a 10% chance of a backslash run of length 1-7. */
static void adv_string(buf_t *b, rng_t *r, int len) {
    putc_(b, '"');
    int w = 0;
    while (w < len && !b->full) {
        if (unif(r) < 0.1) {
            const int k = (int)irange(r, 1, 7);
            for (int i = 0; i < k / 2; i++) puts_(b, "\\\\");
            if (k & 1) puts_(b, (next64(r) & 1) ? "\\\"" : "\\n");
            w += k + 1;
        }
        const char *word = kWords[next64(r) % NWORDS];
        puts_(b, word);
        putc_(b, ' ');
        w += (int)strlen(word) + 1;
    }
    putc_(b, '"');
}

static void adv_number_array(buf_t *b, rng_t *r, int count) {
    putc_(b, '[');
    for (int i = 0; i < count && !b->full; i++) {
        if (i) putc_(b, ',');
        if (next64(r) & 1) {
            put_int(b, irange(r, -100000, 100000));
        } else {
            put_int(b, irange(r, 0, 999));
            putc_(b, '.');
            put_int(b, irange(r, 0, 99));
        }
    }
    putc_(b, ']');
}

/* Nested filler value of `depth` levels and roughly `budget` bytes: a
 * chain/tree of objects and arrays whose leaves are long strings or arrays
 * of at most 1000 numbers. */
static void adv_filler(buf_t *b, rng_t *r, int depth, int64_t budget) {
    if (depth <= 1) {
        if (budget > 6000 || (next64(r) & 1))
            adv_string(b, r, (int)(budget > 16 ? budget : 16));
        else
            adv_number_array(b, r, (int)(budget / 7 > 1000 ? 1000 : budget / 7));
        return;
    }
    const int as_array = next64(r) & 1;
    int kids = (int)irange(r, 1, 3);
    if (budget / kids < 64) kids = 1;
    putc_(b, as_array ? '[' : '{');
    for (int i = 0; i < kids && !b->full; i++) {
        if (i) putc_(b, ',');
        if (!as_array) {
            putc_(b, '"');
            puts_(b, kWords[next64(r) % NWORDS]);
            put_int(b, i);
            puts_(b, "\":");
        }
        adv_filler(b, r, depth - 1, budget / kids);
    }
    putc_(b, as_array ? ']' : '}');
}

static void adversarial(buf_t *b, rng_t *r, int64_t id) {
    const int64_t target = (int64_t)exp(log(100.0) + unif(r) * (log(1048576.0) - log(100.0)));
    const int depth = (int)irange(r, 1, 16);
    /* field order: the queried fields land between filler fields */
    int order[4] = {0, 1, 2, 3};
    for (int i = 3; i > 0; i--) {
        int j = (int)irange(r, 0, i), t = order[i];
        order[i] = order[j];
        order[j] = t;
    }
    puts_(b, "{\"id\":");
    put_int(b, id);
    for (int k = 0; k < 4 && !b->full; k++) {
        putc_(b, ',');
        switch (order[k]) {
            case 0: { /* a.b.c.d, missing at a random level for ~30% */
                const int miss_at = unif(r) < 0.3 ? (int)irange(r, 0, 3) : -1;
                static const char *keys[4] = {"a", "b", "c", "d"};
                int opened = 0;
                for (int l = 0; l < 4; l++) {
                    putc_(b, '"');
                    puts_(b, l == miss_at ? "q" : keys[l]);
                    puts_(b, "\":");
                    if (l < 3) {
                        putc_(b, '{');
                        opened++;
                        if (next64(r) & 1) {
                            puts_(b, "\"s\":");
                            adv_string(b, r, (int)irange(r, 4, 40));
                            putc_(b, ',');
                        }
                    }
                }
                adv_string(b, r, (int)irange(r, 4, 30));
                for (int l = 0; l < opened; l++) putc_(b, '}');
                break;
            }
            case 1: /* arr: ~30% short (0-5 elements, so arr[5] misses) */
                puts_(b, "\"arr\":");
                adv_number_array(b, r, unif(r) < 0.3 ? (int)irange(r, 0, 5) : (int)irange(r, 6, 1000));
                break;
            case 2: { /* x[0].y[2].z */
                puts_(b, "\"x\":[");
                const int nx = unif(r) < 0.1 ? 0 : (int)irange(r, 1, 3);
                for (int i = 0; i < nx; i++) {
                    if (i) putc_(b, ',');
                    puts_(b, "{\"y\":[");
                    const int ny = unif(r) < 0.2 ? (int)irange(r, 0, 2) : (int)irange(r, 3, 6);
                    for (int j = 0; j < ny; j++) {
                        if (j) putc_(b, ',');
                        if (unif(r) < 0.1) {
                            puts_(b, "{\"w\":1}");
                        } else {
                            puts_(b, "{\"z\":");
                            put_int(b, irange(r, 0, 1000));
                            putc_(b, '}');
                        }
                    }
                    puts_(b, "]}");
                }
                putc_(b, ']');
                break;
            }
            default: /* filler of the drawn depth */
                puts_(b, "\"pad\":");
                adv_filler(b, r, depth, target);
                break;
        }
    }
    putc_(b, '}');
}

typedef void (*line_fn)(buf_t *, rng_t *, int64_t, double);

static void tweet_fn(buf_t *b, rng_t *r, int64_t id, double p) { tweet(b, r, id, p); }
static void adv_fn(buf_t *b, rng_t *r, int64_t id, double p) {
    (void)p;
    adversarial(b, r, id);
}

/* Fills out[0, cap) block by block; each block holds whole lines followed by
 * spaces up to the block end when the next line does not fit. */
static int64_t fill(uint8_t *out, int64_t cap, uint64_t seed, line_fn fn, double param, int64_t block) {
    const int64_t nblocks = (cap + block - 1) / block;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t k = 0; k < nblocks; k++) {
        uint8_t *start = out + k * block;
        uint8_t *end = out + (k + 1 < nblocks ? (k + 1) * block : cap);
        rng_t r = {seed * 0x9E3779B97F4A7C15ull ^ (uint64_t)(k + 1) * 0xD1B54A32D192ED03ull};
        int64_t id = 1000000000000ll + k * 100000000ll;
        uint8_t *cur = start;
        for (;;) {
            buf_t b = {cur, end - 1, 0};
            fn(&b, &r, id++, param);
            if (b.full) break;
            *b.p++ = '\n';
            cur = b.p;
        }
        /* pad the rest of the block with a whitespace-only line */
        if (cur < end) {
            memset(cur, ' ', (size_t)(end - cur));
            end[-1] = '\n';
        }
    }
    return cap;
}

GPJGEN_API int64_t gpjgen_tweets(uint8_t *out, int64_t cap, uint64_t seed, double p_empty_hashtags) {
    return fill(out, cap, seed, tweet_fn, p_empty_hashtags, 8 << 20);
}

GPJGEN_API int64_t gpjgen_adversarial(uint8_t *out, int64_t cap, uint64_t seed) {
    return fill(out, cap, seed, adv_fn, 0.0, 64 << 20);
}
