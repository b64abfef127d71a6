// SHA-256 (FIPS 180-4) for the CPU search's two fixed-size messages: the
// 64-byte public key (two blocks, the second the constant padding) and the
// 26-byte name hash || identity hash (one block).  Two compressions: the x86
// SHA extensions (sha256rnds2 / sha256msg1 / sha256msg2) where the CPU has
// them, chosen once at run time, else portable C.
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

}  // namespace cpu_sha
