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

// One step of the bit-matrix transpose: swaps bit rows of a and b at
// distance s (bits of mask m of b with the bits s higher of a).
GPJ_HD void swap_bits(uint32_t& a, uint32_t& b, int s, uint32_t m) {
    const uint32_t t = ((a >> s) ^ b) & m;
    b ^= t;
    a ^= t << s;
}

// Classifies 32 bytes given as 8 little-endian u32 (v[j] = bytes 4j..4j+3).
// The bytes are first transposed so that r[w] holds bytes {w, w+8, w+16,
// w+24}; in each byte lane k they form an 8x8 bit matrix (row w = byte
// 8k+w, column = bit of the byte), transposed in three rounds of swaps so
// that row b afterwards holds bit b of byte 8k+w at bit 8k+w: the eight bit
// planes of the 32 bytes, in byte order.  Each class is then the AND of its
// characters' bit pattern over the planes:
//   '"' 0x22 = 0010 0010   ':' 0x3A = 0011 1010   '\n' 0x0A = 0000 1010
//   ',' 0x2C = 0010 1100   '\\' 0x5C = 0101 1100
//   '[' 0x5B, '{' 0x7B = 01x1 1011 (open)   ']' 0x5D, '}' 0x7D = 01x1 1101 (close)
GPJ_HD void classify32(const uint32_t v[8], uint32_t& bs, uint32_t& qt, uint32_t& nl, uint32_t& op,
                       uint32_t& cl, uint32_t& st, uint32_t& cn) {
    uint32_t r[8];
    transpose4(v[0], v[2], v[4], v[6], r[0], r[1], r[2], r[3]);
    transpose4(v[1], v[3], v[5], v[7], r[4], r[5], r[6], r[7]);
#pragma unroll
    for (int w = 0; w < 4; w++) swap_bits(r[w], r[w + 4], 4, 0x0F0F0F0Fu);
#pragma unroll
    for (int w = 0; w < 8; w += 4) {
        swap_bits(r[w], r[w + 2], 2, 0x33333333u);
        swap_bits(r[w + 1], r[w + 3], 2, 0x33333333u);
    }
#pragma unroll
    for (int w = 0; w < 8; w += 2) swap_bits(r[w], r[w + 1], 1, 0x55555555u);
    const uint32_t p0 = r[0], p1 = r[1], p2 = r[2], p3 = r[3], p4 = r[4], p5 = r[5], p6 = r[6], p7 = r[7];
    const uint32_t row0 = ~(p7 | p6);            // 0x00-0x3F
    const uint32_t row1 = ~p7 & p6;              // 0x40-0x7F
    const uint32_t low010 = ~p2 & p1 & ~p0;      // bits 2-0 = 010
    const uint32_t low100 = p2 & ~(p1 | p0);     // bits 2-0 = 100
    qt = row0 & p5 & ~(p4 | p3) & low010;
    cn = row0 & p5 & p4 & p3 & low010;
    nl = row0 & ~(p5 | p4) & p3 & low010;
    const uint32_t cm = row0 & p5 & ~p4 & p3 & low100;
    bs = row1 & ~p5 & p4 & p3 & low100;
    const uint32_t br = row1 & p4 & p3 & p0;     // bits 1-2 tell open from close
    op = br & ~p2 & p1;
    cl = br & p2 & ~p1;
    st = cm | cn | op | cl;  // ',' ':' and the brackets
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
