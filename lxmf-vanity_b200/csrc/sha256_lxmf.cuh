// The LXMF destination-hash chain on the GPU (sm_100a).
//
//   identity hash = SHA-256(u || ed)[0..16]          64-byte message: 2 blocks
//   destination   = SHA-256(name_hash || ih)[0..16]  26-byte message: 1 block
//
// Same three compressions as the reference's lxmf_address (src/gpu/common.h:
// 221-253) and the CPU path (src/main.rs:179-189), specialised:
//   - block 2 is the fixed padding block of a 64-byte message, so its whole
//     message schedule is a compile-time constant (folded into K + W);
//   - block 3 carries the search's name hash in words 0-2 and zeros in words
//     7-14, so rounds 0 and 1 (which see only the name hash) are done once per
//     search on the host (sha_block3_head) and their zero words fold away;
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

__device__ __forceinline__ uint32_t rotr(uint32_t x, uint32_t n) { return __funnelshift_r(x, x, n); }
__device__ __forceinline__ uint32_t bsig0(uint32_t a) { return rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22); }
__device__ __forceinline__ uint32_t bsig1(uint32_t e) { return rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25); }
__device__ __forceinline__ uint32_t ssig0(uint32_t w) { return rotr(w, 7) ^ rotr(w, 18) ^ (w >> 3); }
__device__ __forceinline__ uint32_t ssig1(uint32_t w) { return rotr(w, 17) ^ rotr(w, 19) ^ (w >> 10); }
__device__ __forceinline__ uint32_t ch(uint32_t e, uint32_t f, uint32_t g) { return (e & f) ^ (~e & g); }
__device__ __forceinline__ uint32_t maj(uint32_t a, uint32_t b, uint32_t c) { return (a & b) | (c & (a | b)); }

// Rounds [R0, 64) of one compression over the 16 message words `w`
// (overwritten by the rolling schedule), with the working state in s[0..7].
// The caller adds the chaining value.
template <int R0>
__device__ __forceinline__ void rounds(uint32_t s[8], uint32_t w[16]) {
    uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
#pragma unroll
    for (int i = R0; i < 64; i++) {
        if (i >= 16) w[i & 15] += ssig0(w[(i - 15) & 15]) + w[(i - 7) & 15] + ssig1(w[(i - 2) & 15]);
        const uint32_t t1 = h + bsig1(e) + ch(e, f, g) + K[i] + w[i & 15];
        const uint32_t t2 = bsig0(a) + maj(a, b, c);
        h = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
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
    uint32_t head[8];   // block-3 working state after rounds 0 and 1 (from IV, nh[0], nh[1])
    uint32_t want[4];   // prefix compare: (dest[k] & mask[k]) == want[k]
    uint32_t mask[4];
};

// Destination hash (4 big-endian words) of a 64-byte public key whose first
// 32 bytes are the little-endian words u[0..7] and whose last 32 bytes are
// the big-endian words hi[0..7].
__device__ __forceinline__ void dest_hash(const uint32_t u[8], const uint32_t hi[8], const AddrConsts& c,
                                          uint32_t out[4]) {
    uint32_t w[16], s[8];
    // Block 1: u (byte-swapped to big-endian words) || Ed25519 key.
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = __byte_perm(u[i], 0, 0x0123);
#pragma unroll
    for (int i = 0; i < 8; i++) w[8 + i] = hi[i];
    s[0] = LXSHA_IV0; s[1] = LXSHA_IV1; s[2] = LXSHA_IV2; s[3] = LXSHA_IV3;
    s[4] = LXSHA_IV4; s[5] = LXSHA_IV5; s[6] = LXSHA_IV6; s[7] = LXSHA_IV7;
    rounds<0>(s, w);
    uint32_t h1[8];
    h1[0] = s[0] + LXSHA_IV0; h1[1] = s[1] + LXSHA_IV1; h1[2] = s[2] + LXSHA_IV2; h1[3] = s[3] + LXSHA_IV3;
    h1[4] = s[4] + LXSHA_IV4; h1[5] = s[5] + LXSHA_IV5; h1[6] = s[6] + LXSHA_IV6; h1[7] = s[7] + LXSHA_IV7;
    // Block 2: the padding block of a 64-byte message (constant schedule).
    w[0] = 0x80000000u;
#pragma unroll
    for (int i = 1; i < 15; i++) w[i] = 0;
    w[15] = 512;
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = h1[i];
    rounds<0>(s, w);
    const uint32_t ih0 = s[0] + h1[0], ih1 = s[1] + h1[1], ih2 = s[2] + h1[2], ih3 = s[3] + h1[3];
    // Block 3: name_hash (10) || identity hash (16) || padding, length 208 bits.
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
#pragma unroll
    for (int i = 0; i < 8; i++) s[i] = c.head[i];
    rounds<2>(s, w);
    out[0] = s[0] + LXSHA_IV0;
    out[1] = s[1] + LXSHA_IV1;
    out[2] = s[2] + LXSHA_IV2;
    out[3] = s[3] + LXSHA_IV3;
}

}  // namespace lxsha
