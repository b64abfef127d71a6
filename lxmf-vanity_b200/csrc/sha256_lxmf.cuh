// The LXMF destination-hash chain on the GPU (sm_100a).
//
//   identity hash = SHA-256(u || ed)[0..16]          64-byte message: 2 blocks
//   destination   = SHA-256(name_hash || ih)[0..16]  26-byte message: 1 block
//
// The three compressions of the reference's lxmf_address (src/gpu/common.h:
// 221-253) and of the CPU path (src/main.rs:179-189).  Code size matters as
// much as instruction count here: the walk kernel keeps tens of warps per SM
// in flight, and a fully unrolled chain (three times 64 rounds) does not fit
// the instruction caches.  So:
//   - rounds run as loops over 16-round unrolled bodies (the 8 working
//     variables rotate statically inside a body, so no moves are needed);
//   - blocks 1 and 3 share one generic compression (a two-pass loop);
//   - block 2, the fixed padding block of a 64-byte message, has a constant
//     message schedule: its rounds read precomputed K + W words (kKW2) and
//     skip the schedule entirely;
//   - only the first four output words are formed: the destination hash.
#pragma once
#include <cstdint>

namespace lxsha {

__device__ __constant__ uint32_t K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

// K[i] + W[i] for the padding block of a 64-byte message
// (W = 0x80000000, 0 x 14, 512, extended by the FIPS 180-4 schedule).
__device__ __constant__ uint32_t kKW2[64] = {
    0xc28a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf374,
    0x649b69c1, 0xf0fe4786, 0x0fe1edc6, 0x240cf254, 0x4fe9346f, 0x6cc984be, 0x61b9411e, 0x16f988fa,
    0xf2c65152, 0xa88e5a6d, 0xb019fc65, 0xb9d99ec7, 0x9a1231c3, 0xe70eeaa0, 0xfdb1232b, 0xc7353eb0,
    0x3069bad5, 0xcb976d5f, 0x5a0f118f, 0xdc1eeefd, 0x0a35b689, 0xde0b7a04, 0x58f4ca9d, 0xe15d5b16,
    0x007f3e86, 0x37088980, 0xa507ea32, 0x6fab9537, 0x17406110, 0x0d8cd6f1, 0xcdaa3b6d, 0xc0bbbe37,
    0x83613bda, 0xdb48a363, 0x0b02e931, 0x6fd15ca7, 0x521afaca, 0x31338431, 0x6ed41a95, 0x6d437890,
    0xc39c91f2, 0x9eccabbd, 0xb5c9a0e6, 0x532fb63c, 0xd2c741c6, 0x07237ea3, 0xa4954b68, 0x4c191d76};

__device__ __forceinline__ uint32_t rotr(uint32_t x, uint32_t n) { return __funnelshift_r(x, x, n); }
__device__ __forceinline__ uint32_t bsig0(uint32_t a) { return rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22); }
__device__ __forceinline__ uint32_t bsig1(uint32_t e) { return rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25); }

// The schedule's sigmas stay on the ALU pipe: moving their right shifts onto
// the IMAD pipe as high-word multiplies by 2^(32-s) was measured slower on
// B200 (the high-word multiply costs more IMAD issue than the shift saves).
__device__ __forceinline__ uint32_t ssig0(uint32_t w) { return rotr(w, 7) ^ rotr(w, 18) ^ (w >> 3); }
__device__ __forceinline__ uint32_t ssig1(uint32_t w) { return rotr(w, 17) ^ rotr(w, 19) ^ (w >> 10); }
__device__ __forceinline__ uint32_t ch(uint32_t e, uint32_t f, uint32_t g) { return (e & f) ^ (~e & g); }
__device__ __forceinline__ uint32_t maj(uint32_t a, uint32_t b, uint32_t c) { return (a & b) | (c & (a | b)); }

// Additions on the multiply-add pipe.  The chain is bound by the integer ALU
// pipe (rotates, LOP3, IADD3) while the IMAD pipe idles, so two-input sums
// off the round's critical path are issued as x * one + y, with `one` a
// runtime 1 (a kernel parameter) that the compiler cannot fold back into an
// IADD3.
__device__ __forceinline__ uint32_t madd(uint32_t x, uint32_t y, uint32_t one) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(one), "r"(y));
    return r;
}

// One round: the new e lands in d and the new a in h (the caller rotates
// names).  Every sum is a two-input IMAD; the ALU pipe keeps only the
// rotates and the LOP3s of Sigma0, Sigma1, Ch and Maj.
#ifndef LXSHA_T1_ON_ALU
#define LXSHA_T1(hk, s1, chv) madd(madd(hk, s1, one), chv, one)
#else
#define LXSHA_T1(hk, s1, chv) ((hk) + (s1) + (chv))
#endif
#define LXSHA_R(a, b, c, d, e, f, g, h, kw)                                \
    {                                                                      \
        const uint32_t hk_ = madd(h, (kw), one);                           \
        const uint32_t t1_ = LXSHA_T1(hk_, bsig1(e), ch(e, f, g));         \
        const uint32_t s0m_ = madd(bsig0(a), maj(a, b, c), one);           \
        d = madd(d, t1_, one);                                             \
        h = madd(t1_, s0m_, one);                                          \
    }

#define LXSHA_SCHED(w, r)                                                                           \
    (w[(r)] = madd(madd(madd(w[(r)], w[((r) + 9) & 15], one), ssig0(w[((r) + 1) & 15]), one),     \
                   ssig1(w[((r) + 14) & 15]), one))

// 16 rounds with message words (SCHED: extend the schedule in place first).
template <bool SCHED>
__device__ __forceinline__ void rounds16(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d, uint32_t& e,
                                         uint32_t& f, uint32_t& g, uint32_t& h, uint32_t w[16], const uint32_t* k,
                                         uint32_t one) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const int r = 8 * half;
        if (SCHED) {
#pragma unroll
            for (int i = 0; i < 8; i++) LXSHA_SCHED(w, r + i);
        }
        LXSHA_R(a, b, c, d, e, f, g, h, madd(w[r + 0], k[r + 0], one));
        LXSHA_R(h, a, b, c, d, e, f, g, madd(w[r + 1], k[r + 1], one));
        LXSHA_R(g, h, a, b, c, d, e, f, madd(w[r + 2], k[r + 2], one));
        LXSHA_R(f, g, h, a, b, c, d, e, madd(w[r + 3], k[r + 3], one));
        LXSHA_R(e, f, g, h, a, b, c, d, madd(w[r + 4], k[r + 4], one));
        LXSHA_R(d, e, f, g, h, a, b, c, madd(w[r + 5], k[r + 5], one));
        LXSHA_R(c, d, e, f, g, h, a, b, madd(w[r + 6], k[r + 6], one));
        LXSHA_R(b, c, d, e, f, g, h, a, madd(w[r + 7], k[r + 7], one));
    }
}

// 16 rounds whose K + W words are given (a constant message).
__device__ __forceinline__ void rounds16_kw(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d, uint32_t& e,
                                            uint32_t& f, uint32_t& g, uint32_t& h, const uint32_t* kw,
                                            uint32_t one) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const int r = 8 * half;
        LXSHA_R(a, b, c, d, e, f, g, h, kw[r + 0]);
        LXSHA_R(h, a, b, c, d, e, f, g, kw[r + 1]);
        LXSHA_R(g, h, a, b, c, d, e, f, kw[r + 2]);
        LXSHA_R(f, g, h, a, b, c, d, e, kw[r + 3]);
        LXSHA_R(e, f, g, h, a, b, c, d, kw[r + 4]);
        LXSHA_R(d, e, f, g, h, a, b, c, kw[r + 5]);
        LXSHA_R(c, d, e, f, g, h, a, b, kw[r + 6]);
        LXSHA_R(b, c, d, e, f, g, h, a, kw[r + 7]);
    }
}

// 64 rounds over message w (overwritten by the schedule); s in, working
// state out (the caller adds the chaining value).
__device__ __forceinline__ void compress(uint32_t s[8], uint32_t w[16], uint32_t one) {
    uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
    rounds16<false>(a, b, c, d, e, f, g, h, w, K, one);
#pragma unroll 1
    for (int j = 1; j < 4; j++) rounds16<true>(a, b, c, d, e, f, g, h, w, K + 16 * j, one);
    s[0] = a; s[1] = b; s[2] = c; s[3] = d; s[4] = e; s[5] = f; s[6] = g; s[7] = h;
}

// 64 rounds of the constant padding block.
__device__ __forceinline__ void compress_pad64(uint32_t s[8], uint32_t one) {
    uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
#pragma unroll 1
    for (int j = 0; j < 4; j++) rounds16_kw(a, b, c, d, e, f, g, h, kKW2 + 16 * j, one);
    s[0] = a; s[1] = b; s[2] = c; s[3] = d; s[4] = e; s[5] = f; s[6] = g; s[7] = h;
}

#define LXSHA_IV0 0x6a09e667u
#define LXSHA_IV1 0xbb67ae85u
#define LXSHA_IV2 0x3c6ef372u
#define LXSHA_IV3 0xa54ff53au
#define LXSHA_IV4 0x510e527fu
#define LXSHA_IV5 0x9b05688cu
#define LXSHA_IV6 0x1f83d9abu
#define LXSHA_IV7 0x5be0cd19u

// Per-search constants of the chain.
struct AddrConsts {
    uint32_t ed[8];     // Ed25519 public key, big-endian words (block-1 words 8..15)
    uint32_t nh[3];     // name hash, big-endian words; nh[2] holds bytes 8, 9 in its top half
    uint32_t want[4];   // prefix compare: (dest[k] & mask[k]) == want[k]
    uint32_t mask[4];
    uint32_t one;       // 1 (see madd)
};

__device__ __forceinline__ void iv(uint32_t s[8]) {
    s[0] = LXSHA_IV0; s[1] = LXSHA_IV1; s[2] = LXSHA_IV2; s[3] = LXSHA_IV3;
    s[4] = LXSHA_IV4; s[5] = LXSHA_IV5; s[6] = LXSHA_IV6; s[7] = LXSHA_IV7;
}

// Destination hash (4 big-endian words) of a 64-byte public key whose first
// 32 bytes are the little-endian words u[0..7] and whose last 32 bytes are
// the big-endian words hi[0..7].  `one` is the runtime 1 of madd: callers
// whose search constants live in shared memory pass it from the kernel
// parameters, so the sums read it from the constant bank (one from shared
// memory cost the pool kernel 4%).
__device__ __forceinline__ void dest_hash_one(const uint32_t u[8], const uint32_t hi[8], const AddrConsts& c,
                                              uint32_t one, uint32_t out[4]) {
    uint32_t w[16], s[8];
    // Block 1: u (byte-swapped to big-endian words) || Ed25519 key.
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = __byte_perm(u[i], 0, 0x0123);
#pragma unroll
    for (int i = 0; i < 8; i++) w[8 + i] = hi[i];
    iv(s);
#pragma unroll 1
    for (int pass = 0;; pass++) {
        compress(s, w, one);
        if (pass == 1) break;
        // Block 2: the padding block, chained from block 1.
        uint32_t h1[8], t[8];
        h1[0] = s[0] + LXSHA_IV0; h1[1] = s[1] + LXSHA_IV1; h1[2] = s[2] + LXSHA_IV2; h1[3] = s[3] + LXSHA_IV3;
        h1[4] = s[4] + LXSHA_IV4; h1[5] = s[5] + LXSHA_IV5; h1[6] = s[6] + LXSHA_IV6; h1[7] = s[7] + LXSHA_IV7;
#pragma unroll
        for (int i = 0; i < 8; i++) t[i] = h1[i];
        compress_pad64(t, one);
        const uint32_t ih0 = t[0] + h1[0], ih1 = t[1] + h1[1], ih2 = t[2] + h1[2], ih3 = t[3] + h1[3];
        // Block 3: name_hash (10) || identity hash (16) || padding, 208 bits.
        w[0] = c.nh[0];
        w[1] = c.nh[1];
        w[2] = c.nh[2] | (ih0 >> 16);
        w[3] = __funnelshift_l(ih1, ih0, 16);
        w[4] = __funnelshift_l(ih2, ih1, 16);
        w[5] = __funnelshift_l(ih3, ih2, 16);
        w[6] = (ih3 << 16) | 0x8000u;
#pragma unroll
        for (int i = 7; i < 15; i++) w[i] = 0;
        w[15] = 26 * 8;
        iv(s);
    }
    out[0] = s[0] + LXSHA_IV0;
    out[1] = s[1] + LXSHA_IV1;
    out[2] = s[2] + LXSHA_IV2;
    out[3] = s[3] + LXSHA_IV3;
}

__device__ __forceinline__ void dest_hash(const uint32_t u[8], const uint32_t hi[8], const AddrConsts& c,
                                          uint32_t out[4]) {
    dest_hash_one(u, hi, c, c.one, out);
}

}  // namespace lxsha
