// SHA-256 (FIPS 180-4) for the CPU search's two fixed-size messages: the
// 64-byte public key (two blocks, the second the constant padding) and the
// 26-byte name hash || identity hash (one block).  Three implementations,
// chosen at run time: AVX-512F sixteen messages at a time (namespace x16),
// the x86 SHA extensions (sha256rnds2 / sha256msg1 / sha256msg2), one or two
// messages at a time, and portable C.
#pragma once

#include <cstdint>
#include <cstring>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace cpu_sha {

constexpr uint32_t K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

constexpr uint32_t IV[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                            0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

// One compression of the 64-byte block `p` into `s`, portable C.
inline void compress_c(uint32_t s[8], const uint8_t* p) {
    uint32_t w[64];
    for (int i = 0; i < 16; i++)
        w[i] = (uint32_t)p[4 * i] << 24 | (uint32_t)p[4 * i + 1] << 16 | (uint32_t)p[4 * i + 2] << 8 | p[4 * i + 3];
    for (int i = 16; i < 64; i++) {
        const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
        const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
    for (int i = 0; i < 64; i++) {
        const uint32_t t1 = h + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + K[i] + w[i];
        const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
        h = g;
        g = f;
        f = e;
        e = d + t1;
        d = c;
        c = b;
        b = a;
        a = t1 + t2;
    }
    s[0] += a;
    s[1] += b;
    s[2] += c;
    s[3] += d;
    s[4] += e;
    s[5] += f;
    s[6] += g;
    s[7] += h;
}

#if defined(__x86_64__)
// One compression with the SHA extensions.  The state travels as two
// registers, (A, B, E, F) and (C, D, G, H), highest dword first, the order
// sha256rnds2 takes them in; each sha256rnds2 runs two rounds.
__attribute__((target("sha,sse4.1"))) inline void compress_ni(uint32_t s[8], const uint8_t* p) {
    const __m128i bswap = _mm_set_epi64x(0x0c0d0e0f08090a0bll, 0x0405060700010203ll);
    __m128i t = _mm_loadu_si128((const __m128i*)&s[0]);   // a b c d
    __m128i cdgh = _mm_loadu_si128((const __m128i*)&s[4]);  // e f g h
    t = _mm_shuffle_epi32(t, 0xB1);                          // b a d c
    cdgh = _mm_shuffle_epi32(cdgh, 0x1B);                    // h g f e
    __m128i abef = _mm_alignr_epi8(t, cdgh, 8);              // f e b a
    cdgh = _mm_blend_epi16(cdgh, t, 0xF0);                   // h g d c
    const __m128i abef0 = abef, cdgh0 = cdgh;
    __m128i m[16];
    for (int i = 0; i < 4; i++) m[i] = _mm_shuffle_epi8(_mm_loadu_si128((const __m128i*)(p + 16 * i)), bswap);
    for (int i = 4; i < 16; i++) {
        // W[t..t+3] = sigma1 terms + W[t-7..t-4] + sigma0 terms + W[t-16..t-13].
        const __m128i x = _mm_add_epi32(_mm_sha256msg1_epu32(m[i - 4], m[i - 3]), _mm_alignr_epi8(m[i - 1], m[i - 2], 4));
        m[i] = _mm_sha256msg2_epu32(x, m[i - 1]);
    }
    for (int i = 0; i < 16; i++) {
        __m128i wk = _mm_add_epi32(m[i], _mm_loadu_si128((const __m128i*)&K[4 * i]));
        cdgh = _mm_sha256rnds2_epu32(cdgh, abef, wk);
        wk = _mm_shuffle_epi32(wk, 0x0E);
        abef = _mm_sha256rnds2_epu32(abef, cdgh, wk);
    }
    abef = _mm_add_epi32(abef, abef0);
    cdgh = _mm_add_epi32(cdgh, cdgh0);
    t = _mm_shuffle_epi32(abef, 0x1B);                                   // a b e f
    cdgh = _mm_shuffle_epi32(cdgh, 0xB1);                                // g h c d
    _mm_storeu_si128((__m128i*)&s[0], _mm_blend_epi16(t, cdgh, 0xF0));   // a b c d
    _mm_storeu_si128((__m128i*)&s[4], _mm_alignr_epi8(cdgh, t, 8));      // e f g h
}

// Two compressions at once: two independent blocks into two states, their
// instructions interleaved so that one stream's sha256rnds2 latency hides
// behind the other's.  The schedule is kept as a rolling window of four
// message vectors per stream (twelve XMM registers in all).
__attribute__((target("sha,sse4.1"))) inline void compress_ni2(uint32_t s0[8], const uint8_t* p0, uint32_t s1[8],
                                                              const uint8_t* p1) {
    const __m128i bswap = _mm_set_epi64x(0x0c0d0e0f08090a0bll, 0x0405060700010203ll);
    uint32_t* st[2] = {s0, s1};
    const uint8_t* pp[2] = {p0, p1};
    __m128i abef[2], cdgh[2], abef0[2], cdgh0[2], m[2][4];
    for (int j = 0; j < 2; j++) {
        __m128i t = _mm_shuffle_epi32(_mm_loadu_si128((const __m128i*)&st[j][0]), 0xB1);
        __m128i c = _mm_shuffle_epi32(_mm_loadu_si128((const __m128i*)&st[j][4]), 0x1B);
        abef[j] = _mm_alignr_epi8(t, c, 8);
        cdgh[j] = _mm_blend_epi16(c, t, 0xF0);
        abef0[j] = abef[j];
        cdgh0[j] = cdgh[j];
        for (int i = 0; i < 4; i++) m[j][i] = _mm_shuffle_epi8(_mm_loadu_si128((const __m128i*)(pp[j] + 16 * i)), bswap);
    }
    for (int i = 0; i < 16; i++) {
        const __m128i k = _mm_loadu_si128((const __m128i*)&K[4 * i]);
        for (int j = 0; j < 2; j++) {
            __m128i w;
            if (i < 4) {
                w = m[j][i];
            } else {
                // W[4i..4i+3] from the last four vectors (slot i & 3 holds W[4(i-4)..]).
                const __m128i x = _mm_add_epi32(_mm_sha256msg1_epu32(m[j][i & 3], m[j][(i + 1) & 3]),
                                                _mm_alignr_epi8(m[j][(i + 3) & 3], m[j][(i + 2) & 3], 4));
                w = _mm_sha256msg2_epu32(x, m[j][(i + 3) & 3]);
                m[j][i & 3] = w;
            }
            __m128i wk = _mm_add_epi32(w, k);
            cdgh[j] = _mm_sha256rnds2_epu32(cdgh[j], abef[j], wk);
            wk = _mm_shuffle_epi32(wk, 0x0E);
            abef[j] = _mm_sha256rnds2_epu32(abef[j], cdgh[j], wk);
        }
    }
    for (int j = 0; j < 2; j++) {
        const __m128i a = _mm_add_epi32(abef[j], abef0[j]), c = _mm_add_epi32(cdgh[j], cdgh0[j]);
        const __m128i t = _mm_shuffle_epi32(a, 0x1B);
        const __m128i u = _mm_shuffle_epi32(c, 0xB1);
        _mm_storeu_si128((__m128i*)&st[j][0], _mm_blend_epi16(t, u, 0xF0));
        _mm_storeu_si128((__m128i*)&st[j][4], _mm_alignr_epi8(u, t, 8));
    }
}

inline bool have_sha_ni() {
    static const bool yes = __builtin_cpu_supports("sha") && __builtin_cpu_supports("sse4.1");
    return yes;
}
#endif

template <bool NI>
inline void compress(uint32_t s[8], const uint8_t* p) {
#if defined(__x86_64__)
    if (NI) {
        compress_ni(s, p);
        return;
    }
#endif
    compress_c(s, p);
}

// The padding block of a 64-byte message: 0x80, zeros, bit length 512.
inline const uint8_t* pad64() {
    static const uint8_t b[64] = {0x80, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                  0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                  0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0x02, 0x00};
    return b;
}

// The LXMF address (lxmf_address, main.rs:180-189): the first 16 bytes of
// SHA-256(name_hash || SHA-256(x_pub || ed_pub)[0..16]).  `pk` holds x_pub
// then ed_pub; `block` is a 64-byte buffer whose bytes 0..9 hold the name
// hash and whose padding (0x80 at 26, bit length 208 at 62..63, zeros
// between) the caller set once.
template <bool NI>
inline void address(const uint8_t pk[64], uint8_t block[64], uint8_t out[16]) {
    uint32_t s[8];
    memcpy(s, IV, sizeof s);
    compress<NI>(s, pk);
    compress<NI>(s, pad64());
    for (int i = 0; i < 4; i++) {
        block[10 + 4 * i] = (uint8_t)(s[i] >> 24);
        block[11 + 4 * i] = (uint8_t)(s[i] >> 16);
        block[12 + 4 * i] = (uint8_t)(s[i] >> 8);
        block[13 + 4 * i] = (uint8_t)s[i];
    }
    memcpy(s, IV, sizeof s);
    compress<NI>(s, block);
    for (int i = 0; i < 4; i++) {
        out[4 * i] = (uint8_t)(s[i] >> 24);
        out[4 * i + 1] = (uint8_t)(s[i] >> 16);
        out[4 * i + 2] = (uint8_t)(s[i] >> 8);
        out[4 * i + 3] = (uint8_t)s[i];
    }
}

#if defined(__x86_64__)
// address() for two public keys at once with the SHA extensions.  `blocks`
// is two 64-byte buffers, each set up by address_block.
inline void address2_ni(const uint8_t pk0[64], const uint8_t pk1[64], uint8_t blocks[2][64], uint8_t out0[16],
                        uint8_t out1[16]) {
    uint32_t s0[8], s1[8];
    memcpy(s0, IV, sizeof s0);
    memcpy(s1, IV, sizeof s1);
    compress_ni2(s0, pk0, s1, pk1);
    compress_ni2(s0, pad64(), s1, pad64());
    uint32_t* st[2] = {s0, s1};
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < 4; i++) {
            blocks[j][10 + 4 * i] = (uint8_t)(st[j][i] >> 24);
            blocks[j][11 + 4 * i] = (uint8_t)(st[j][i] >> 16);
            blocks[j][12 + 4 * i] = (uint8_t)(st[j][i] >> 8);
            blocks[j][13 + 4 * i] = (uint8_t)st[j][i];
        }
    memcpy(s0, IV, sizeof s0);
    memcpy(s1, IV, sizeof s1);
    compress_ni2(s0, blocks[0], s1, blocks[1]);
    uint8_t* out[2] = {out0, out1};
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < 4; i++) {
            out[j][4 * i] = (uint8_t)(st[j][i] >> 24);
            out[j][4 * i + 1] = (uint8_t)(st[j][i] >> 16);
            out[j][4 * i + 2] = (uint8_t)(st[j][i] >> 8);
            out[j][4 * i + 3] = (uint8_t)st[j][i];
        }
}
#endif

// Sets up the second hash's block: name hash and padding.
inline void address_block(const uint8_t nh[10], uint8_t block[64]) {
    memset(block, 0, 64);
    memcpy(block, nh, 10);
    block[26] = 0x80;
    block[62] = 0x00;
    block[63] = 208;  // 26 bytes = 208 bits
}

// K[i] + W[i] of the 64-byte message's padding block, whose schedule is a
// constant (0x80000000, zeros, bit length 512).
struct PadKW {
    uint32_t kw[64];
    constexpr PadKW() : kw() {
        uint32_t w[64] = {};
        w[0] = 0x80000000u;
        w[15] = 512;
        for (int i = 16; i < 64; i++) {
            const uint32_t x = w[i - 15], y = w[i - 2];
            const uint32_t s0 = ((x >> 7) | (x << 25)) ^ ((x >> 18) | (x << 14)) ^ (x >> 3);
            const uint32_t s1 = ((y >> 17) | (y << 15)) ^ ((y >> 19) | (y << 13)) ^ (y >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        for (int i = 0; i < 64; i++) kw[i] = K[i] + w[i];
    }
};
constexpr PadKW PAD_KW{};

// ---- Sixteen keys that share one ed_pub and one name hash (a walker's keys).
// Block 1's words 8..15 (ed_pub) and block 3's words 0, 1 (name hash) and
// 7..15 (zeros, length) are the same for every key, so what depends on them
// alone is computed once, in scalar code: block 1's first round, the K + W of
// its rounds 8..15 and the constant parts of its schedule words 16..31; block
// 3's first two rounds and the constant parts of its words 16..31.

inline uint32_t s_ssig0(uint32_t x) { return rotr(x, 7) ^ rotr(x, 18) ^ (x >> 3); }
inline uint32_t s_ssig1(uint32_t x) { return rotr(x, 17) ^ rotr(x, 19) ^ (x >> 10); }

struct Shared16 {
    uint32_t t1c, t2c;  // block 1, round 0: T1 = t1c + W0, T2 = t2c
    uint32_t kw1[8];    // block 1: K[8 + i] + W[8 + i]
    uint32_t c1[16];    // block 1: the ed_pub-only part of W[16 + i]
    uint32_t s3[8];     // block 3: the state after rounds 0 and 1
    uint32_t nh2;       // block 3: W2's name-hash half
    uint32_t c3_16, c3_17, c3_18, c3_30, c3_31;
};

inline void shared16_init(const uint8_t ed[32], const uint8_t nh[10], Shared16* c) {
    uint32_t e[8];
    for (int i = 0; i < 8; i++)
        e[i] = (uint32_t)ed[4 * i] << 24 | (uint32_t)ed[4 * i + 1] << 16 | (uint32_t)ed[4 * i + 2] << 8 | ed[4 * i + 3];
    auto bsig0 = [](uint32_t a) { return rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22); };
    auto bsig1 = [](uint32_t x) { return rotr(x, 6) ^ rotr(x, 11) ^ rotr(x, 25); };
    auto ch = [](uint32_t x, uint32_t y, uint32_t z) { return (x & y) ^ (~x & z); };
    auto maj = [](uint32_t x, uint32_t y, uint32_t z) { return (x & y) ^ (x & z) ^ (y & z); };
    c->t1c = IV[7] + bsig1(IV[4]) + ch(IV[4], IV[5], IV[6]) + K[0];
    c->t2c = bsig0(IV[0]) + maj(IV[0], IV[1], IV[2]);
    for (int i = 0; i < 8; i++) c->kw1[i] = K[8 + i] + e[i];
    // W16 = s1(W14) + W9 + s0(W1) + W0, ...: the terms in W8..W15 = e0..e7.
    c->c1[0] = s_ssig1(e[6]) + e[1];
    c->c1[1] = s_ssig1(e[7]) + e[2];
    for (int i = 2; i < 7; i++) c->c1[i] = e[i + 1];  // W18..W22: W11..W15
    c->c1[7] = s_ssig0(e[0]);                         // W23: s0(W8)
    for (int i = 8; i < 15; i++) c->c1[i] = s_ssig0(e[i - 7]) + e[i - 8];  // W24..W30: s0(W9..W15) + W8..W14
    c->c1[15] = e[7];                                                       // W31: W15
    // Block 3: name_hash[0..9] || identity hash || 0x80 || zeros || 208.
    const uint32_t n0 = (uint32_t)nh[0] << 24 | (uint32_t)nh[1] << 16 | (uint32_t)nh[2] << 8 | nh[3];
    const uint32_t n1 = (uint32_t)nh[4] << 24 | (uint32_t)nh[5] << 16 | (uint32_t)nh[6] << 8 | nh[7];
    c->nh2 = (uint32_t)nh[8] << 24 | (uint32_t)nh[9] << 16;
    uint32_t s[8];
    memcpy(s, IV, sizeof s);
    const uint32_t w01[2] = {n0, n1};
    for (int r = 0; r < 2; r++) {
        const uint32_t t1 = s[7] + bsig1(s[4]) + ch(s[4], s[5], s[6]) + K[r] + w01[r];
        const uint32_t t2 = bsig0(s[0]) + maj(s[0], s[1], s[2]);
        memmove(s + 1, s, 7 * sizeof(uint32_t));
        s[4] += t1;
        s[0] = t1 + t2;
    }
    memcpy(c->s3, s, sizeof s);
    c->c3_16 = s_ssig0(n1) + n0;
    c->c3_17 = s_ssig1(208) + n1;
    c->c3_18 = s_ssig1(c->c3_16);
    c->c3_30 = s_ssig0(208);
    c->c3_31 = s_ssig0(c->c3_16) + 208;
}

#if defined(__x86_64__)
// Sixteen addresses at once with AVX-512F: message m in 32-bit lane m of each
// vector.  A rotate is one vprord, and Sigma0 / Sigma1 / sigma0 / sigma1's
// three-way XOR, Ch and Maj are one vpternlogd each, so a round is about 16
// vector instructions for 16 keys.
namespace x16 {

typedef __m512i V;
#define LXCPU_X16 __attribute__((target("avx512f")))

LXCPU_X16 inline V add(V a, V b) { return _mm512_add_epi32(a, b); }
LXCPU_X16 inline V xor3(V a, V b, V c) { return _mm512_ternarylogic_epi32(a, b, c, 0x96); }
LXCPU_X16 inline V bsig0(V a) { return xor3(_mm512_ror_epi32(a, 2), _mm512_ror_epi32(a, 13), _mm512_ror_epi32(a, 22)); }
LXCPU_X16 inline V bsig1(V e) { return xor3(_mm512_ror_epi32(e, 6), _mm512_ror_epi32(e, 11), _mm512_ror_epi32(e, 25)); }
LXCPU_X16 inline V ssig0(V w) { return xor3(_mm512_ror_epi32(w, 7), _mm512_ror_epi32(w, 18), _mm512_srli_epi32(w, 3)); }
LXCPU_X16 inline V ssig1(V w) { return xor3(_mm512_ror_epi32(w, 17), _mm512_ror_epi32(w, 19), _mm512_srli_epi32(w, 10)); }
LXCPU_X16 inline V ch(V e, V f, V g) { return _mm512_ternarylogic_epi32(e, f, g, 0xCA); }   // e ? f : g
LXCPU_X16 inline V maj(V a, V b, V c) { return _mm512_ternarylogic_epi32(a, b, c, 0xE8); }  // majority
// Big-endian word of four little-endian bytes: bytes 3 and 1 from the rotate
// right by 8, bytes 2 and 0 from the rotate left.
LXCPU_X16 inline V bswap(V x) {
    return _mm512_ternarylogic_epi32(_mm512_ror_epi32(x, 8), _mm512_rol_epi32(x, 8), _mm512_set1_epi32((int)0xFF00FF00),
                                     0xE4);
}

// One round; the new e lands in d and the new a in h (the caller rotates names).
#define LXCPU_X16_ROUND(a, b, c, d, e, f, g, h, kw)                 \
    {                                                              \
        const V t1_ = add(add(h, kw), add(bsig1(e), ch(e, f, g))); \
        d = add(d, t1_);                                           \
        h = add(t1_, add(bsig0(a), maj(a, b, c)));                 \
    }

// One compression of the 16-word blocks w (schedule extended in place).
LXCPU_X16 __attribute__((always_inline)) inline void compress(V s[8], V w[16]) {
    V a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
#pragma GCC unroll 8
    for (int r = 0; r < 64; r += 8) {
        if (r >= 16) {
#pragma GCC unroll 8
            for (int j = 0; j < 8; j++) {
                const int i = (r + j) & 15;
                w[i] = add(add(w[i], ssig0(w[(i + 1) & 15])), add(w[(i + 9) & 15], ssig1(w[(i + 14) & 15])));
            }
        }
        const int q = r & 15;
        LXCPU_X16_ROUND(a, b, c, d, e, f, g, h, add(w[q + 0], _mm512_set1_epi32((int)K[r + 0])));
        LXCPU_X16_ROUND(h, a, b, c, d, e, f, g, add(w[q + 1], _mm512_set1_epi32((int)K[r + 1])));
        LXCPU_X16_ROUND(g, h, a, b, c, d, e, f, add(w[q + 2], _mm512_set1_epi32((int)K[r + 2])));
        LXCPU_X16_ROUND(f, g, h, a, b, c, d, e, add(w[q + 3], _mm512_set1_epi32((int)K[r + 3])));
        LXCPU_X16_ROUND(e, f, g, h, a, b, c, d, add(w[q + 4], _mm512_set1_epi32((int)K[r + 4])));
        LXCPU_X16_ROUND(d, e, f, g, h, a, b, c, add(w[q + 5], _mm512_set1_epi32((int)K[r + 5])));
        LXCPU_X16_ROUND(c, d, e, f, g, h, a, b, add(w[q + 6], _mm512_set1_epi32((int)K[r + 6])));
        LXCPU_X16_ROUND(b, c, d, e, f, g, h, a, add(w[q + 7], _mm512_set1_epi32((int)K[r + 7])));
    }
    s[0] = add(s[0], a);
    s[1] = add(s[1], b);
    s[2] = add(s[2], c);
    s[3] = add(s[3], d);
    s[4] = add(s[4], e);
    s[5] = add(s[5], f);
    s[6] = add(s[6], g);
    s[7] = add(s[7], h);
}

// The padding block's compression: its K + W are the constants PAD_KW.
LXCPU_X16 __attribute__((always_inline)) inline void compress_pad64(V s[8]) {
    V a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
#pragma GCC unroll 8
    for (int r = 0; r < 64; r += 8) {
        LXCPU_X16_ROUND(a, b, c, d, e, f, g, h, _mm512_set1_epi32((int)PAD_KW.kw[r + 0]));
        LXCPU_X16_ROUND(h, a, b, c, d, e, f, g, _mm512_set1_epi32((int)PAD_KW.kw[r + 1]));
        LXCPU_X16_ROUND(g, h, a, b, c, d, e, f, _mm512_set1_epi32((int)PAD_KW.kw[r + 2]));
        LXCPU_X16_ROUND(f, g, h, a, b, c, d, e, _mm512_set1_epi32((int)PAD_KW.kw[r + 3]));
        LXCPU_X16_ROUND(e, f, g, h, a, b, c, d, _mm512_set1_epi32((int)PAD_KW.kw[r + 4]));
        LXCPU_X16_ROUND(d, e, f, g, h, a, b, c, _mm512_set1_epi32((int)PAD_KW.kw[r + 5]));
        LXCPU_X16_ROUND(c, d, e, f, g, h, a, b, _mm512_set1_epi32((int)PAD_KW.kw[r + 6]));
        LXCPU_X16_ROUND(b, c, d, e, f, g, h, a, _mm512_set1_epi32((int)PAD_KW.kw[r + 7]));
    }
    s[0] = add(s[0], a);
    s[1] = add(s[1], b);
    s[2] = add(s[2], c);
    s[3] = add(s[3], d);
    s[4] = add(s[4], e);
    s[5] = add(s[5], f);
    s[6] = add(s[6], g);
    s[7] = add(s[7], h);
}
#undef LXCPU_X16_ROUND

// The first four big-endian words of the addresses of 16 public keys.  Key m's
// x_pub is the 32 bytes at x + m * x_stride; its ed_pub the 32 bytes at
// ed + m * ed_stride (ed_stride 0: one ed_pub for all).  nh: the name hash.
LXCPU_X16 inline void address16(const uint8_t* x, int x_stride, const uint8_t* ed, int ed_stride, const uint8_t nh[10],
                                V out[4]) {
    const V lane = _mm512_set_epi32(15, 14, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1, 0);
    const V xoff = _mm512_mullo_epi32(lane, _mm512_set1_epi32(x_stride));
    V w[16], s[8];
    for (int j = 0; j < 8; j++) w[j] = bswap(_mm512_i32gather_epi32(xoff, (const void*)(x + 4 * j), 1));
    if (ed_stride) {
        const V eoff = _mm512_mullo_epi32(lane, _mm512_set1_epi32(ed_stride));
        for (int j = 0; j < 8; j++) w[8 + j] = bswap(_mm512_i32gather_epi32(eoff, (const void*)(ed + 4 * j), 1));
    } else {
        for (int j = 0; j < 8; j++) {
            const uint8_t* p = ed + 4 * j;
            w[8 + j] = _mm512_set1_epi32((int)((uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]));
        }
    }
    for (int i = 0; i < 8; i++) s[i] = _mm512_set1_epi32((int)IV[i]);
    compress(s, w);
    compress_pad64(s);
    // Second hash: name_hash (10 bytes) || identity hash (16 bytes), 0x80, length 208.
    const uint32_t nh0 = (uint32_t)nh[0] << 24 | (uint32_t)nh[1] << 16 | (uint32_t)nh[2] << 8 | nh[3];
    const uint32_t nh1 = (uint32_t)nh[4] << 24 | (uint32_t)nh[5] << 16 | (uint32_t)nh[6] << 8 | nh[7];
    const uint32_t nh2 = (uint32_t)nh[8] << 24 | (uint32_t)nh[9] << 16;
    w[0] = _mm512_set1_epi32((int)nh0);
    w[1] = _mm512_set1_epi32((int)nh1);
    w[2] = _mm512_or_si512(_mm512_set1_epi32((int)nh2), _mm512_srli_epi32(s[0], 16));
    w[3] = _mm512_or_si512(_mm512_slli_epi32(s[0], 16), _mm512_srli_epi32(s[1], 16));
    w[4] = _mm512_or_si512(_mm512_slli_epi32(s[1], 16), _mm512_srli_epi32(s[2], 16));
    w[5] = _mm512_or_si512(_mm512_slli_epi32(s[2], 16), _mm512_srli_epi32(s[3], 16));
    w[6] = _mm512_or_si512(_mm512_slli_epi32(s[3], 16), _mm512_set1_epi32(0x8000));
    for (int j = 7; j < 15; j++) w[j] = _mm512_setzero_si512();
    w[15] = _mm512_set1_epi32(208);
    for (int i = 0; i < 8; i++) s[i] = _mm512_set1_epi32((int)IV[i]);
    compress(s, w);
    for (int i = 0; i < 4; i++) out[i] = s[i];
}

// The 16 addresses as bytes: out + 16 * m for key m.
LXCPU_X16 inline void address16_bytes(const uint8_t* x, int x_stride, const uint8_t* ed, int ed_stride,
                                      const uint8_t nh[10], uint8_t* out) {
    V h[4];
    address16(x, x_stride, ed, ed_stride, nh, h);
    alignas(64) uint32_t words[4][16];
    for (int i = 0; i < 4; i++) _mm512_store_si512((void*)words[i], h[i]);
    for (int m = 0; m < 16; m++)
        for (int i = 0; i < 4; i++) {
            out[16 * m + 4 * i] = (uint8_t)(words[i][m] >> 24);
            out[16 * m + 4 * i + 1] = (uint8_t)(words[i][m] >> 16);
            out[16 * m + 4 * i + 2] = (uint8_t)(words[i][m] >> 8);
            out[16 * m + 4 * i + 3] = (uint8_t)words[i][m];
        }
}

// Bit m set where key m's address matches: (word[i] & mask[i]) == want[i] for
// the big-endian prefix words with a nonzero mask (want already masked).
LXCPU_X16 inline uint32_t match16(const uint8_t* x, int x_stride, const uint8_t* ed, const uint8_t nh[10],
                                  const uint32_t want[4], const uint32_t mask[4]) {
    V h[4];
    address16(x, x_stride, ed, 0, nh, h);
    __mmask16 m = 0xFFFF;
    for (int i = 0; i < 4; i++)
        if (mask[i])
            m &= _mm512_cmpeq_epi32_mask(_mm512_and_si512(h[i], _mm512_set1_epi32((int)mask[i])),
                                         _mm512_set1_epi32((int)want[i]));
    return m;
}

#define LXCPU_X16_ROUND(a, b, c, d, e, f, g, h, kw)                 \
    {                                                              \
        const V t1_ = add(add(h, kw), add(bsig1(e), ch(e, f, g))); \
        d = add(d, t1_);                                           \
        h = add(t1_, add(bsig0(a), maj(a, b, c)));                 \
    }
#define LXCPU_X16_K(r) _mm512_set1_epi32((int)K[r])
#define LXCPU_X16_C(x) _mm512_set1_epi32((int)(x))

// Rounds 16..63 with w[i & 15] = W_i for i = 16..31; the names are those of
// round 16 (the caller's state after round 15).
LXCPU_X16 __attribute__((always_inline)) inline void rounds_16_63(V& a, V& b, V& c, V& d, V& e, V& f, V& g, V& h, V w[16]) {
#pragma GCC unroll 6
    for (int r = 16; r < 64; r += 8) {
        if (r >= 32) {
#pragma GCC unroll 8
            for (int j = 0; j < 8; j++) {
                const int i = (r + j) & 15;
                w[i] = add(add(w[i], ssig0(w[(i + 1) & 15])), add(w[(i + 9) & 15], ssig1(w[(i + 14) & 15])));
            }
        }
        const int q = r & 15;
        LXCPU_X16_ROUND(a, b, c, d, e, f, g, h, add(w[q + 0], LXCPU_X16_K(r + 0)));
        LXCPU_X16_ROUND(h, a, b, c, d, e, f, g, add(w[q + 1], LXCPU_X16_K(r + 1)));
        LXCPU_X16_ROUND(g, h, a, b, c, d, e, f, add(w[q + 2], LXCPU_X16_K(r + 2)));
        LXCPU_X16_ROUND(f, g, h, a, b, c, d, e, add(w[q + 3], LXCPU_X16_K(r + 3)));
        LXCPU_X16_ROUND(e, f, g, h, a, b, c, d, add(w[q + 4], LXCPU_X16_K(r + 4)));
        LXCPU_X16_ROUND(d, e, f, g, h, a, b, c, add(w[q + 5], LXCPU_X16_K(r + 5)));
        LXCPU_X16_ROUND(c, d, e, f, g, h, a, b, add(w[q + 6], LXCPU_X16_K(r + 6)));
        LXCPU_X16_ROUND(b, c, d, e, f, g, h, a, add(w[q + 7], LXCPU_X16_K(r + 7)));
    }
}

// Block 1 (x_pub words x[0..7], the shared ed_pub in c) from the initial state:
// s = IV + the compression.
LXCPU_X16 __attribute__((always_inline)) inline void block1_shared(const V x[8], const Shared16& k, V s[8]) {
    // Round 0 on the constant initial state; the names are then round 1's.
    const V t1 = add(x[0], LXCPU_X16_C(k.t1c));
    V h = add(t1, LXCPU_X16_C(k.t2c)), d = add(t1, LXCPU_X16_C(IV[3]));
    V a = LXCPU_X16_C(IV[0]), b = LXCPU_X16_C(IV[1]), c = LXCPU_X16_C(IV[2]);
    V e = LXCPU_X16_C(IV[4]), f = LXCPU_X16_C(IV[5]), g = LXCPU_X16_C(IV[6]);
    LXCPU_X16_ROUND(h, a, b, c, d, e, f, g, add(x[1], LXCPU_X16_K(1)));
    LXCPU_X16_ROUND(g, h, a, b, c, d, e, f, add(x[2], LXCPU_X16_K(2)));
    LXCPU_X16_ROUND(f, g, h, a, b, c, d, e, add(x[3], LXCPU_X16_K(3)));
    LXCPU_X16_ROUND(e, f, g, h, a, b, c, d, add(x[4], LXCPU_X16_K(4)));
    LXCPU_X16_ROUND(d, e, f, g, h, a, b, c, add(x[5], LXCPU_X16_K(5)));
    LXCPU_X16_ROUND(c, d, e, f, g, h, a, b, add(x[6], LXCPU_X16_K(6)));
    LXCPU_X16_ROUND(b, c, d, e, f, g, h, a, add(x[7], LXCPU_X16_K(7)));
    LXCPU_X16_ROUND(a, b, c, d, e, f, g, h, LXCPU_X16_C(k.kw1[0]));
    LXCPU_X16_ROUND(h, a, b, c, d, e, f, g, LXCPU_X16_C(k.kw1[1]));
    LXCPU_X16_ROUND(g, h, a, b, c, d, e, f, LXCPU_X16_C(k.kw1[2]));
    LXCPU_X16_ROUND(f, g, h, a, b, c, d, e, LXCPU_X16_C(k.kw1[3]));
    LXCPU_X16_ROUND(e, f, g, h, a, b, c, d, LXCPU_X16_C(k.kw1[4]));
    LXCPU_X16_ROUND(d, e, f, g, h, a, b, c, LXCPU_X16_C(k.kw1[5]));
    LXCPU_X16_ROUND(c, d, e, f, g, h, a, b, LXCPU_X16_C(k.kw1[6]));
    LXCPU_X16_ROUND(b, c, d, e, f, g, h, a, LXCPU_X16_C(k.kw1[7]));
    // W16..W31: x-dependent terms plus the constant parts.
    V w[16];
    w[0] = add(add(LXCPU_X16_C(k.c1[0]), ssig0(x[1])), x[0]);
    w[1] = add(add(LXCPU_X16_C(k.c1[1]), ssig0(x[2])), x[1]);
    for (int i = 2; i < 7; i++)
        w[i] = add(add(LXCPU_X16_C(k.c1[i]), ssig1(w[i - 2])), add(ssig0(x[i + 1]), x[i]));
    w[7] = add(add(LXCPU_X16_C(k.c1[7]), ssig1(w[5])), add(w[0], x[7]));
    for (int i = 8; i < 15; i++) w[i] = add(add(LXCPU_X16_C(k.c1[i]), ssig1(w[i - 2])), w[i - 7]);
    w[15] = add(add(LXCPU_X16_C(k.c1[15]), ssig1(w[13])), add(w[8], ssig0(w[0])));
    rounds_16_63(a, b, c, d, e, f, g, h, w);
    s[0] = add(a, LXCPU_X16_C(IV[0]));
    s[1] = add(b, LXCPU_X16_C(IV[1]));
    s[2] = add(c, LXCPU_X16_C(IV[2]));
    s[3] = add(d, LXCPU_X16_C(IV[3]));
    s[4] = add(e, LXCPU_X16_C(IV[4]));
    s[5] = add(f, LXCPU_X16_C(IV[5]));
    s[6] = add(g, LXCPU_X16_C(IV[6]));
    s[7] = add(h, LXCPU_X16_C(IV[7]));
}

// Block 3 from the identity hash words ih[0..3]: the first four words of the
// destination hash.
LXCPU_X16 __attribute__((always_inline)) inline void block3_shared(const V ih[4], const Shared16& k, V out[4]) {
    const V y2 = _mm512_or_si512(LXCPU_X16_C(k.nh2), _mm512_srli_epi32(ih[0], 16));
    const V y3 = _mm512_or_si512(_mm512_slli_epi32(ih[0], 16), _mm512_srli_epi32(ih[1], 16));
    const V y4 = _mm512_or_si512(_mm512_slli_epi32(ih[1], 16), _mm512_srli_epi32(ih[2], 16));
    const V y5 = _mm512_or_si512(_mm512_slli_epi32(ih[2], 16), _mm512_srli_epi32(ih[3], 16));
    const V y6 = _mm512_or_si512(_mm512_slli_epi32(ih[3], 16), LXCPU_X16_C(0x8000));
    // The state after rounds 0 and 1, under round 2's names.
    V g = LXCPU_X16_C(k.s3[0]), h = LXCPU_X16_C(k.s3[1]), a = LXCPU_X16_C(k.s3[2]), b = LXCPU_X16_C(k.s3[3]);
    V c = LXCPU_X16_C(k.s3[4]), d = LXCPU_X16_C(k.s3[5]), e = LXCPU_X16_C(k.s3[6]), f = LXCPU_X16_C(k.s3[7]);
    LXCPU_X16_ROUND(g, h, a, b, c, d, e, f, add(y2, LXCPU_X16_K(2)));
    LXCPU_X16_ROUND(f, g, h, a, b, c, d, e, add(y3, LXCPU_X16_K(3)));
    LXCPU_X16_ROUND(e, f, g, h, a, b, c, d, add(y4, LXCPU_X16_K(4)));
    LXCPU_X16_ROUND(d, e, f, g, h, a, b, c, add(y5, LXCPU_X16_K(5)));
    LXCPU_X16_ROUND(c, d, e, f, g, h, a, b, add(y6, LXCPU_X16_K(6)));
    LXCPU_X16_ROUND(b, c, d, e, f, g, h, a, LXCPU_X16_K(7));  // W7..W14 = 0
    LXCPU_X16_ROUND(a, b, c, d, e, f, g, h, LXCPU_X16_K(8));
    LXCPU_X16_ROUND(h, a, b, c, d, e, f, g, LXCPU_X16_K(9));
    LXCPU_X16_ROUND(g, h, a, b, c, d, e, f, LXCPU_X16_K(10));
    LXCPU_X16_ROUND(f, g, h, a, b, c, d, e, LXCPU_X16_K(11));
    LXCPU_X16_ROUND(e, f, g, h, a, b, c, d, LXCPU_X16_K(12));
    LXCPU_X16_ROUND(d, e, f, g, h, a, b, c, LXCPU_X16_K(13));
    LXCPU_X16_ROUND(c, d, e, f, g, h, a, b, LXCPU_X16_K(14));
    LXCPU_X16_ROUND(b, c, d, e, f, g, h, a, LXCPU_X16_C(K[15] + 208u));  // W15 = 208
    V w[16];
    w[0] = LXCPU_X16_C(k.c3_16);
    w[1] = add(LXCPU_X16_C(k.c3_17), ssig0(y2));
    w[2] = add(add(LXCPU_X16_C(k.c3_18), ssig0(y3)), y2);
    w[3] = add(add(ssig1(w[1]), ssig0(y4)), y3);
    w[4] = add(add(ssig1(w[2]), ssig0(y5)), y4);
    w[5] = add(add(ssig1(w[3]), ssig0(y6)), y5);
    w[6] = add(add(ssig1(w[4]), LXCPU_X16_C(208)), y6);
    w[7] = add(ssig1(w[5]), w[0]);
    for (int i = 8; i < 14; i++) w[i] = add(ssig1(w[i - 2]), w[i - 7]);
    w[14] = add(add(ssig1(w[12]), w[7]), LXCPU_X16_C(k.c3_30));
    w[15] = add(add(ssig1(w[13]), w[8]), LXCPU_X16_C(k.c3_31));
    rounds_16_63(a, b, c, d, e, f, g, h, w);
    out[0] = add(a, LXCPU_X16_C(IV[0]));
    out[1] = add(b, LXCPU_X16_C(IV[1]));
    out[2] = add(c, LXCPU_X16_C(IV[2]));
    out[3] = add(d, LXCPU_X16_C(IV[3]));
}
#undef LXCPU_X16_ROUND
#undef LXCPU_X16_K
#undef LXCPU_X16_C

// The first four destination-hash words of 16 keys that share the ed_pub and
// name hash in k, from their x_pub words (big-endian, one key per lane).
LXCPU_X16 __attribute__((always_inline)) inline void address16_shared_core(const V xw[8], const Shared16& k, V out[4]) {
    V s[8];
    block1_shared(xw, k, s);
    compress_pad64(s);
    block3_shared(s, k, out);
}

// address16 for 16 keys that share the ed_pub and name hash in k.
LXCPU_X16 inline void address16_shared(const uint8_t* x, int x_stride, const Shared16& k, V out[4]) {
    const V lane = _mm512_set_epi32(15, 14, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1, 0);
    const V xoff = _mm512_mullo_epi32(lane, _mm512_set1_epi32(x_stride));
    V xw[8];
    for (int j = 0; j < 8; j++) xw[j] = bswap(_mm512_i32gather_epi32(xoff, (const void*)(x + 4 * j), 1));
    address16_shared_core(xw, k, out);
}

LXCPU_X16 inline void address16_shared_bytes(const uint8_t* x, int x_stride, const Shared16& k, uint8_t* out) {
    V h[4];
    address16_shared(x, x_stride, k, h);
    alignas(64) uint32_t words[4][16];
    for (int i = 0; i < 4; i++) _mm512_store_si512((void*)words[i], h[i]);
    for (int m = 0; m < 16; m++)
        for (int i = 0; i < 4; i++) {
            out[16 * m + 4 * i] = (uint8_t)(words[i][m] >> 24);
            out[16 * m + 4 * i + 1] = (uint8_t)(words[i][m] >> 16);
            out[16 * m + 4 * i + 2] = (uint8_t)(words[i][m] >> 8);
            out[16 * m + 4 * i + 3] = (uint8_t)words[i][m];
        }
}

// match16 for keys sharing the ed_pub and name hash in k.
LXCPU_X16 inline uint32_t match16_shared(const uint8_t* x, int x_stride, const Shared16& k, const uint32_t want[4],
                                         const uint32_t mask[4]) {
    V h[4];
    address16_shared(x, x_stride, k, h);
    __mmask16 m = 0xFFFF;
    for (int i = 0; i < 4; i++)
        if (mask[i])
            m &= _mm512_cmpeq_epi32_mask(_mm512_and_si512(h[i], _mm512_set1_epi32((int)mask[i])),
                                         _mm512_set1_epi32((int)want[i]));
    return m;
}

// match16_shared with x_pub stored word-major: word j (little-endian) of key m
// at words[j * stride + m], as the IFMA walk writes its keys; no gathers.
LXCPU_X16 inline uint32_t match16_shared_words(const uint32_t* words, size_t stride, const Shared16& k,
                                               const uint32_t want[4], const uint32_t mask[4]) {
    V xw[8], h[4];
    for (int j = 0; j < 8; j++) xw[j] = bswap(_mm512_loadu_si512((const void*)(words + j * stride)));
    address16_shared_core(xw, k, h);
    __mmask16 m = 0xFFFF;
    for (int i = 0; i < 4; i++)
        if (mask[i])
            m &= _mm512_cmpeq_epi32_mask(_mm512_and_si512(h[i], _mm512_set1_epi32((int)mask[i])),
                                         _mm512_set1_epi32((int)want[i]));
    return m;
}

inline bool available() {
    static const bool yes = __builtin_cpu_supports("avx512f");
    return yes;
}

#undef LXCPU_X16
}  // namespace x16
#endif

}  // namespace cpu_sha
