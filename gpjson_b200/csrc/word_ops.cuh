// Per-64-byte-word bit arithmetic of the structural index.
//
// One "word" is 64 input bytes and the matching bit of every 64-bit bitmap
// (the reference's bitmaps are long[ceil(n/64)], bit i%64 of word i/64 =
// byte i; Sequential.java:40-50).  All functions are __host__ __device__ so
// the same code can be exercised on the CPU by the test suite.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define GPJ_HD __host__ __device__ __forceinline__
#else
#define GPJ_HD inline
#endif

namespace gpj {

// Byte permute: result byte i is byte (s_i & 7) of the 8-byte pair (y:x)
// for the selector nibbles s_i (bit 3 of each nibble ignored).
GPJ_HD uint32_t byte_perm(uint32_t x, uint32_t y, uint32_t s) {
#ifdef __CUDA_ARCH__
    return __byte_perm(x, y, s);
#else
    const uint64_t v = (static_cast<uint64_t>(y) << 32) | x;
    uint32_t r = 0;
    for (int i = 0; i < 4; i++) r |= static_cast<uint32_t>((v >> (8 * ((s >> (4 * i)) & 7))) & 0xFF) << (8 * i);
    return r;
#endif
}

// The same with bit 3 of a selector nibble honoured as PTX prmt's default
// mode defines it: that result byte is the selected byte's bit 7 replicated
// over all eight bits (a zero byte for a table byte below 0x80).
GPJ_HD uint32_t byte_perm_sign(uint32_t x, uint32_t y, uint32_t s) {
#ifdef __CUDA_ARCH__
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(y), "r"(s));
    return r;
#else
    const uint64_t v = (static_cast<uint64_t>(y) << 32) | x;
    uint32_t r = 0;
    for (int i = 0; i < 4; i++) {
        const uint32_t sel = (s >> (4 * i)) & 0xF;
        uint32_t b = static_cast<uint32_t>((v >> (8 * (sel & 7))) & 0xFF);
        if (sel & 8) b = (b & 0x80) ? 0xFF : 0x00;
        r |= b << (8 * i);
    }
    return r;
#endif
}

GPJ_HD int popc64(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __popcll(x);
#else
    return __builtin_popcountll(x);
#endif
}

GPJ_HD int ctz64(uint64_t x) {  // x != 0
#ifdef __CUDA_ARCH__
    return __ffsll(static_cast<long long>(x)) - 1;
#else
    return __builtin_ctzll(x);
#endif
}

GPJ_HD int clz64(uint64_t x) {  // x != 0
#ifdef __CUDA_ARCH__
    return __clzll(static_cast<long long>(x));
#else
    return __builtin_clzll(x);
#endif
}

GPJ_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) >> 32);
#endif
}

// 0x80 in every byte of x equal to the byte replicated in `pattern`
// (pattern bytes < 0x80), 0 elsewhere.  Exact for all 256 byte values:
// the low seven bits are compared with a carry-free add, bit 7 must be 0.
GPJ_HD uint32_t low_differs(uint32_t x, uint32_t pattern) {
    // bit 7 of each byte: the low seven bits of x and pattern differ there
    return ((x ^ pattern) & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
}

GPJ_HD uint32_t eq_bytes(uint32_t x, uint32_t pattern) { return ~(low_differs(x, pattern) | x) & 0x80808080u; }

// 4x4 byte transpose of rows r0..r3: column c = {r0.b_c, r1.b_c, r2.b_c, r3.b_c}.
GPJ_HD void transpose4(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3, uint32_t& c0,
                       uint32_t& c1, uint32_t& c2, uint32_t& c3) {
    const uint32_t a = byte_perm(r0, r1, 0x5140), b = byte_perm(r0, r1, 0x7362);
    const uint32_t c = byte_perm(r2, r3, 0x5140), d = byte_perm(r2, r3, 0x7362);
    c0 = byte_perm(a, c, 0x5410);
    c1 = byte_perm(a, c, 0x7632);
    c2 = byte_perm(b, d, 0x5410);
    c3 = byte_perm(b, d, 0x7632);
}

// Character classes of one 64-byte word, one bit per byte.
struct ClassMasks {
    uint64_t backslash;   // '\\'
    uint64_t quote;       // '"'
    uint64_t newline;     // '\n'
    uint64_t open;        // '{' '['
    uint64_t close;       // '}' ']'
    uint64_t structural;  // '{' '[' '}' ']' ':' ','
    uint64_t colon;       // ':'
};

// Class bits of each byte of 32 bytes: the byte's high nibble h and low
// nibble l look up one table each (PRMT with 4-bit selectors) and the
// results AND together, so a class bit survives only for the (h, l) pairs
// of its characters: '\n' 0A, ',' 2C, ':' 3A, '\\' 5C, '[' 5B and '{' 7B
// (open), ']' 5D and '}' 7D (close).  Lookups are by h (0-7; a non-ASCII
// byte, h >= 8, reads a sign-replicated zero) and by l ^ 8 (the low nibbles
// A-D of these characters become 2-5; every other value either selects a
// zero entry or reads a sign-replicated zero; byte_perm_sign).  '"' is the one character
// with a low nibble below 8 and is found by a byte compare (bit 7).
constexpr uint32_t kClsNewline = 1u << 0, kClsComma = 1u << 1, kClsColon = 1u << 2, kClsBackslash = 1u << 3,
                   kClsOpen = 1u << 4, kClsClose = 1u << 5, kClsQuote = 1u << 7;
// table by high nibble: entries 0-3 and 4-7
constexpr uint32_t kHiTab0 = kClsNewline | (0u << 8) | (kClsComma << 16) | (kClsColon << 24);
constexpr uint32_t kHiTab1 = 0u | ((kClsBackslash | kClsOpen | kClsClose) << 8) | (0u << 16) |
                             ((kClsOpen | kClsClose) << 24);
// table by low nibble ^ 8: entries 0-3 (l = 8, 9, A, B) and 4-7 (l = C, D, E, F)
constexpr uint32_t kLoTab0 = 0u | (0u << 8) | ((kClsNewline | kClsColon) << 16) | (kClsOpen << 24);
constexpr uint32_t kLoTab1 = (kClsComma | kClsBackslash) | (kClsClose << 8) | (0u << 16) | (0u << 24);

// The four nibbles at bits 0-3, 8-11, 16-19, 24-27 of x packed into a PRMT
// selector (bits 0-15).
GPJ_HD uint32_t nibble_selector(uint32_t x) {
    const uint32_t c = (x | (x >> 4)) & 0x00FF00FFu;
    return byte_perm(c, 0, 0x3320);
}

GPJ_HD uint32_t class_bytes(uint32_t x) {
    const uint32_t hi = nibble_selector((x >> 4) & 0x0F0F0F0Fu);
    const uint32_t lo = nibble_selector((x ^ 0x08080808u) & 0x0F0F0F0Fu);
    const uint32_t c = byte_perm_sign(kHiTab0, kHiTab1, hi) & byte_perm_sign(kLoTab0, kLoTab1, lo);
    return c | eq_bytes(x, 0x22222222u);  // '"' at bit 7
}

// One step of the bit-matrix transpose: swaps bit rows of a and b at
// distance s (bits of mask m of b with the bits s higher of a).
GPJ_HD void swap_bits(uint32_t& a, uint32_t& b, int s, uint32_t m) {
    const uint32_t t = ((a >> s) ^ b) & m;
    b ^= t;
    a ^= t << s;
}

// Classifies 32 bytes given as 8 little-endian u32 (v[j] = bytes 4j..4j+3).
// The bytes are first transposed so that t[w] holds bytes {w, w+8, w+16,
// w+24}; their class bytes form, in each byte lane k, an 8x8 bit matrix
// (row w = t[w]'s class byte, column = class bit), transposed in three
// rounds of swaps so that row c afterwards holds class c with byte 8k+w at
// bit 8k+w: the class masks in byte order.
GPJ_HD void classify32(const uint32_t v[8], uint32_t& bs, uint32_t& qt, uint32_t& nl, uint32_t& op,
                       uint32_t& cl, uint32_t& st, uint32_t& cn) {
    uint32_t t[8];
    transpose4(v[0], v[2], v[4], v[6], t[0], t[1], t[2], t[3]);
    transpose4(v[1], v[3], v[5], v[7], t[4], t[5], t[6], t[7]);
    uint32_t r[8];
#pragma unroll
    for (int w = 0; w < 8; w++) r[w] = class_bytes(t[w]);
#pragma unroll
    for (int w = 0; w < 4; w++) swap_bits(r[w], r[w + 4], 4, 0x0F0F0F0Fu);
#pragma unroll
    for (int w = 0; w < 8; w += 4) {
        swap_bits(r[w], r[w + 2], 2, 0x33333333u);
        swap_bits(r[w + 1], r[w + 3], 2, 0x33333333u);
    }
#pragma unroll
    for (int w = 0; w < 8; w += 2) swap_bits(r[w], r[w + 1], 1, 0x55555555u);
    nl = r[0];
    cn = r[2];
    bs = r[3];
    op = r[4];
    cl = r[5];
    qt = r[7];
    st = r[1] | r[2] | op | cl;  // ',' ':' and the brackets
}

GPJ_HD ClassMasks classify64(const uint32_t v[16]) {
    uint32_t b0, q0, n0, o0, c0, s0, k0, b1, q1, n1, o1, c1, s1, k1;
    classify32(v, b0, q0, n0, o0, c0, s0, k0);
    classify32(v + 8, b1, q1, n1, o1, c1, s1, k1);
    ClassMasks m;
    m.backslash = (static_cast<uint64_t>(b1) << 32) | b0;
    m.quote = (static_cast<uint64_t>(q1) << 32) | q0;
    m.newline = (static_cast<uint64_t>(n1) << 32) | n0;
    m.open = (static_cast<uint64_t>(o1) << 32) | o0;
    m.close = (static_cast<uint64_t>(c1) << 32) | c0;
    m.structural = (static_cast<uint64_t>(s1) << 32) | s0;
    m.colon = (static_cast<uint64_t>(k1) << 32) | k0;
    return m;
}

// Escaped positions of a word.  The reference's rule (Sequential.java:44-56)
// is: byte i is escaped iff the run of backslashes ending at byte i-1 has odd
// length.  `carry_in` is that parity for the word's first byte.
//
// Runs are found with additions: adding a run's start bit to the backslash
// mask carries through the run and leaves exactly the bit after it.  Runs
// starting on an even bit end escaped on an odd bit and vice versa, so runs
// are split by start parity.  A run continuing from the previous word acts
// like a run starting at bit 0 (carry_in = 0) or at bit -1 (carry_in = 1).
// Returns the escaped mask; *carry_out is the parity for the next word.
GPJ_HD uint64_t escaped_mask(uint64_t bs, uint32_t carry_in, uint32_t* carry_out) {
    const uint64_t kEven = 0x5555555555555555ull, kOdd = ~kEven;
    const uint64_t starts = bs & ~(bs << 1);
    const uint64_t first = carry_in ? (bs & 1u) : 0;  // run continuing with odd phase
    const uint64_t even_starts = (starts & kEven) & ~first;
    const uint64_t odd_starts = (starts & kOdd) | first;
    const uint64_t even_sum = bs + even_starts;
    const uint64_t odd_sum = bs + odd_starts;
    *carry_out = odd_sum < bs ? 1u : 0u;
    uint64_t esc = ((even_sum & ~bs) & kOdd) | ((odd_sum & ~bs) & kEven);
    // Byte 0 after an odd run that ended in the previous word.
    if (carry_in && !(bs & 1u)) esc |= 1u;
    return esc;
}

// Inclusive prefix XOR: bit i = XOR of bits 0..i (in-string state after
// byte i, CombinedIndex's create_string_index does the same per word).
GPJ_HD uint64_t prefix_xor(uint64_t x) {
    x ^= x << 1;
    x ^= x << 2;
    x ^= x << 4;
    x ^= x << 8;
    x ^= x << 16;
    x ^= x << 32;
    return x;
}

// Word summary composed across words and tiles.  Given the state before a
// span (s = inside a string, d = level counter, nl = newlines so far), the
// state after it is
//   s' = s ^ q,  d' = d + (s ? ddt - dd0 : dd0),  nl' = nl + nl_count
// where dd0 is the span's net depth change when it starts outside a string
// and ddt its raw open-minus-close count (starting inside a string flips
// every in-string bit of the span, which turns dd0 into ddt - dd0).
struct Span {
    int32_t q;    // quote parity
    int32_t dd0;  // depth change when entered outside a string
    int32_t ddt;  // open - close ignoring strings
    int32_t nl;   // newline count
};

GPJ_HD Span span_identity() { return Span{0, 0, 0, 0}; }

// a then b.
GPJ_HD Span span_compose(const Span& a, const Span& b) {
    Span r;
    r.q = a.q ^ b.q;
    r.dd0 = a.dd0 + (a.q ? b.ddt - b.dd0 : b.dd0);
    r.ddt = a.ddt + b.ddt;
    r.nl = a.nl + b.nl;
    return r;
}

// Structural bits of one word split by level.  `open`, `close`, `structural`
// are already restricted to bytes outside strings; `depth` is the level
// counter before the word's first byte (it starts at -1 at the beginning of
// the file, LeveledBitmapsIndex.java:73-82).  Rules of Sequential.java:88-101:
// an opening bracket increments the counter and is marked at the new level,
// a closing bracket is marked at the current level and then decrements it,
// ':' and ',' are marked at the current level.  Levels outside
// [0, num_levels) are not marked.
//
// The word is cut into segments of constant level: an opening bracket at
// byte x starts a segment at x, a closing bracket at byte x ends one after
// x, so the cuts are `open | close << 1` and crossing the cut at x changes
// the level by open[x] - close[x-1] (a '}' directly followed by '{' cuts
// once with no change).  Every cut costs the same straight-line work, so
// the lanes of a warp stay converged whatever brackets their words hold.
// A word changes the level by at most 64, so the level is carried in 32
// bits with `depth` clamped to +-128: a clamped start is out of range for
// every byte exactly when the true one is.  Returns the level after the word.
template <int LV>
GPJ_HD int64_t split_levels(uint64_t open, uint64_t close, uint64_t structural, int64_t depth,
                            uint64_t (&lv)[LV]) {
#pragma unroll
    for (int k = 0; k < LV; k++) lv[k] = 0;
    const uint64_t close_after = close << 1;
    uint64_t cuts = open | close_after;
    uint64_t rest = structural;
    int d = depth > 128 ? 128 : (depth < -128 ? -128 : static_cast<int>(depth));
    while (cuts) {
        const uint64_t cut = cuts & (~cuts + 1);  // lowest cut
        const uint64_t seg = rest & (cut - 1);    // the bytes before it
        rest ^= seg;
#pragma unroll
        for (int k = 0; k < LV; k++)
            if (d == k) lv[k] |= seg;
        d += ((open & cut) ? 1 : 0) - ((close_after & cut) ? 1 : 0);
        cuts ^= cut;
    }
#pragma unroll
    for (int k = 0; k < LV; k++)
        if (d == k) lv[k] |= rest;
    return depth + popc64(open) - popc64(close);
}

}  // namespace gpj
