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
// dest_hash_one is the general chain (any 64-byte public key: the primitive
// microbench).  The walks use dest_hash_folded (at the end of this file),
// which takes a search's Ed25519-key-only work out of the per-key chain.
#pragma once
#include <cstdint>

namespace lxsha {

// FIPS 180-4 round constants (the initializer is shared with the host-side fold_chain).
#define LXSHA_K_INIT {  \
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,  \
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,  \
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,  \
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,  \
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,  \
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,  \
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,  \
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2}

__device__ __constant__ uint32_t K[64] = LXSHA_K_INIT;

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

// ---- The folded chain: the walks' hashing, with a search's constants folded in.
//
// In the walks every key of a search hashes the same Ed25519 key (block-1
// message words 8..15) and the same name hash; block 3's words 7..15 are the
// zero padding and the length.  So each of blocks 1 and 3 has message words
// 8..15 fixed per search, and whatever depends only on them is computed once
// on the host (fold_chain) instead of once per key:
//   - the K + W words of rounds 8..15;
//   - in schedule words 16..31, the sigma0 of words 8..15 (in words 23..30),
//     the sigma1 of words 14 and 15 (in words 16 and 17) and the plain words
//     8..15: one constant addend per schedule word.
// That is 10 sigma functions (about 40 ALU-pipe operations) per block.
// Block 2's K + W words are constant.  All twelve 16-round passes of the
// chain run through one loop whose body is one of three bodies (message words
// 0..7 plus a K + W table; the first schedule extension with the addends; the
// generic schedule extension), so that the code stays about as small as the
// unfolded chain's.

// Per search: K + W of the table passes (words 0..7 of a block-1 or block-3
// pass hold K alone, its message words being added at run time; block 2's
// passes hold its K + W), and the schedule addends of blocks 1 and 3.
struct ChainConsts {
    uint32_t kw[6][16];  // [0] block 1 rounds 0..15, [1] block 3 rounds 0..15, [2 + j] block 2 rounds 16j..16j+15
    uint32_t sc[2][16];  // [0] block 1, [1] block 3: constant part of schedule words 16..31
};

// Host: the folded constants of a search whose Ed25519 key is the
// big-endian words ed[0..7].
inline void fold_chain(const uint32_t ed[8], ChainConsts& cc) {
    static const uint32_t k[64] = LXSHA_K_INIT;
    auto rot = [](uint32_t x, int n) { return (x >> n) | (x << (32 - n)); };
    auto s0 = [&](uint32_t x) { return rot(x, 7) ^ rot(x, 18) ^ (x >> 3); };
    auto s1 = [&](uint32_t x) { return rot(x, 17) ^ rot(x, 19) ^ (x >> 10); };
    // Block 2: the padding block of a 64-byte message, scheduled in full.
    uint32_t w2[64] = {0x80000000u};
    w2[15] = 512;
    for (int t = 16; t < 64; t++) w2[t] = s1(w2[t - 2]) + w2[t - 7] + s0(w2[t - 15]) + w2[t - 16];
    for (int j = 0; j < 4; j++)
        for (int r = 0; r < 16; r++) cc.kw[2 + j][r] = k[16 * j + r] + w2[16 * j + r];
    for (int b = 0; b < 2; b++) {
        // Message words 8..15: the Ed25519 key (block 1), or zeros and the
        // bit length of the 26-byte message (block 3).
        uint32_t m[16] = {0};
        for (int i = 0; i < 8; i++) m[8 + i] = b == 0 ? ed[i] : 0;
        if (b == 1) m[15] = 26 * 8;
        for (int r = 0; r < 16; r++) cc.kw[b][r] = k[r] + m[r];  // m[0..7] = 0: words 0..7 are added per key
        uint32_t* c = cc.sc[b];
        c[0] = m[9] + s1(m[14]);
        c[1] = m[10] + s1(m[15]);
        for (int i = 2; i <= 6; i++) c[i] = m[i + 9];
        c[7] = s0(m[8]);
        for (int i = 8; i <= 14; i++) c[i] = m[i] + s0(m[i + 1]);
        c[15] = m[15];
    }
}

// 16 rounds of a table pass: K + W is w[r] + T[r] for rounds 0..7 (T = K, or
// block 2's K + W with w[0..7] = 0) and T[r] for rounds 8..15.
__device__ __forceinline__ void rounds16_tab(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d, uint32_t& e,
                                             uint32_t& f, uint32_t& g, uint32_t& h, const uint32_t w[16],
                                             const uint32_t* T, uint32_t one) {
    LXSHA_R(a, b, c, d, e, f, g, h, madd(w[0], T[0], one));
    LXSHA_R(h, a, b, c, d, e, f, g, madd(w[1], T[1], one));
    LXSHA_R(g, h, a, b, c, d, e, f, madd(w[2], T[2], one));
    LXSHA_R(f, g, h, a, b, c, d, e, madd(w[3], T[3], one));
    LXSHA_R(e, f, g, h, a, b, c, d, madd(w[4], T[4], one));
    LXSHA_R(d, e, f, g, h, a, b, c, madd(w[5], T[5], one));
    LXSHA_R(c, d, e, f, g, h, a, b, madd(w[6], T[6], one));
    LXSHA_R(b, c, d, e, f, g, h, a, madd(w[7], T[7], one));
    LXSHA_R(a, b, c, d, e, f, g, h, T[8]);
    LXSHA_R(h, a, b, c, d, e, f, g, T[9]);
    LXSHA_R(g, h, a, b, c, d, e, f, T[10]);
    LXSHA_R(f, g, h, a, b, c, d, e, T[11]);
    LXSHA_R(e, f, g, h, a, b, c, d, T[12]);
    LXSHA_R(d, e, f, g, h, a, b, c, T[13]);
    LXSHA_R(c, d, e, f, g, h, a, b, T[14]);
    LXSHA_R(b, c, d, e, f, g, h, a, T[15]);
}

// Rounds 16..31 of block 1 or 3, with schedule words 16..31 built from
// w[0..7] (message words 0..7) and the addends sc (message words 8..15 are
// folded in and never read).  w[i] becomes word 16 + i.
__device__ __forceinline__ void rounds16_sched1(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d, uint32_t& e,
                                                uint32_t& f, uint32_t& g, uint32_t& h, uint32_t w[16],
                                                const uint32_t* sc, uint32_t one) {
    w[0] = madd(madd(w[0], ssig0(w[1]), one), sc[0], one);
    w[1] = madd(madd(w[1], ssig0(w[2]), one), sc[1], one);
#pragma unroll
    for (int i = 2; i <= 6; i++) w[i] = madd(madd(madd(w[i], ssig0(w[i + 1]), one), ssig1(w[i - 2]), one), sc[i], one);
    w[7] = madd(madd(madd(w[7], w[0], one), ssig1(w[5]), one), sc[7], one);
    LXSHA_R(a, b, c, d, e, f, g, h, madd(w[0], K[16], one));
    LXSHA_R(h, a, b, c, d, e, f, g, madd(w[1], K[17], one));
    LXSHA_R(g, h, a, b, c, d, e, f, madd(w[2], K[18], one));
    LXSHA_R(f, g, h, a, b, c, d, e, madd(w[3], K[19], one));
    LXSHA_R(e, f, g, h, a, b, c, d, madd(w[4], K[20], one));
    LXSHA_R(d, e, f, g, h, a, b, c, madd(w[5], K[21], one));
    LXSHA_R(c, d, e, f, g, h, a, b, madd(w[6], K[22], one));
    LXSHA_R(b, c, d, e, f, g, h, a, madd(w[7], K[23], one));
#pragma unroll
    for (int i = 8; i <= 14; i++) w[i] = madd(madd(w[i - 7], ssig1(w[i - 2]), one), sc[i], one);
    w[15] = madd(madd(madd(w[8], ssig1(w[13]), one), ssig0(w[0]), one), sc[15], one);
    LXSHA_R(a, b, c, d, e, f, g, h, madd(w[8], K[24], one));
    LXSHA_R(h, a, b, c, d, e, f, g, madd(w[9], K[25], one));
    LXSHA_R(g, h, a, b, c, d, e, f, madd(w[10], K[26], one));
    LXSHA_R(f, g, h, a, b, c, d, e, madd(w[11], K[27], one));
    LXSHA_R(e, f, g, h, a, b, c, d, madd(w[12], K[28], one));
    LXSHA_R(d, e, f, g, h, a, b, c, madd(w[13], K[29], one));
    LXSHA_R(c, d, e, f, g, h, a, b, madd(w[14], K[30], one));
    LXSHA_R(b, c, d, e, f, g, h, a, madd(w[15], K[31], one));
}

// Destination hash (4 big-endian words) of the public key whose first 32
// bytes are the little-endian words u[0..7] and whose last 32 bytes are the
// search's Ed25519 key folded into cc (fold_chain); nh is the search's name
// hash (AddrConsts::nh).  Passes p = 0..11 of 16 rounds: 0..3 block 1,
// 4..7 block 2, 8..11 block 3.  `one` as in dest_hash_one.
__device__ __forceinline__ void dest_hash_folded(const uint32_t u[8], const ChainConsts& cc, const uint32_t nh[3],
                                                 uint32_t one, uint32_t out[4]) {
    uint32_t w[16], h1[8];
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = __byte_perm(u[i], 0, 0x0123);
#pragma unroll
    for (int i = 8; i < 16; i++) w[i] = 0;
    uint32_t a = LXSHA_IV0, b = LXSHA_IV1, c = LXSHA_IV2, d = LXSHA_IV3;
    uint32_t e = LXSHA_IV4, f = LXSHA_IV5, g = LXSHA_IV6, h = LXSHA_IV7;
#pragma unroll 1
    for (int p = 0; p < 12; p++) {
        const int q = p & 3;
        const bool pad = (p >> 2) == 1;
        if (pad || q == 0) {
            rounds16_tab(a, b, c, d, e, f, g, h, w, cc.kw[pad ? 2 + q : (p >> 3)], one);
        } else if (q == 1) {
            rounds16_sched1(a, b, c, d, e, f, g, h, w, cc.sc[p >> 3], one);
        } else {
            rounds16<true>(a, b, c, d, e, f, g, h, w, K + 16 * q, one);
        }
        if (p == 3) {
            // Block 1 done: chain into block 2 (the padding block, no message words).
            h1[0] = a + LXSHA_IV0; h1[1] = b + LXSHA_IV1; h1[2] = c + LXSHA_IV2; h1[3] = d + LXSHA_IV3;
            h1[4] = e + LXSHA_IV4; h1[5] = f + LXSHA_IV5; h1[6] = g + LXSHA_IV6; h1[7] = h + LXSHA_IV7;
            a = h1[0]; b = h1[1]; c = h1[2]; d = h1[3]; e = h1[4]; f = h1[5]; g = h1[6]; h = h1[7];
#pragma unroll
            for (int i = 0; i < 8; i++) w[i] = 0;
        } else if (p == 7) {
            // Identity hash = the first 4 words; block 3: name_hash (10) || ih (16) || padding.
            const uint32_t ih0 = a + h1[0], ih1 = b + h1[1], ih2 = c + h1[2], ih3 = d + h1[3];
            w[0] = nh[0];
            w[1] = nh[1];
            w[2] = nh[2] | (ih0 >> 16);
            w[3] = __funnelshift_l(ih1, ih0, 16);
            w[4] = __funnelshift_l(ih2, ih1, 16);
            w[5] = __funnelshift_l(ih3, ih2, 16);
            w[6] = (ih3 << 16) | 0x8000u;
            w[7] = 0;
            a = LXSHA_IV0; b = LXSHA_IV1; c = LXSHA_IV2; d = LXSHA_IV3;
            e = LXSHA_IV4; f = LXSHA_IV5; g = LXSHA_IV6; h = LXSHA_IV7;
        }
    }
    out[0] = a + LXSHA_IV0;
    out[1] = b + LXSHA_IV1;
    out[2] = c + LXSHA_IV2;
    out[3] = d + LXSHA_IV3;
}

}  // namespace lxsha
