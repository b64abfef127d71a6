/*
 * CPU oracle for the lxmf-vanity key-walk search.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls
 * this file: it is the checker that the CUDA path is compared against, and
 * the timed CPU restatement ("port") that bench.py reports beside the GPU.
 *
 * It restates, in plain C written from the mathematics, the reference's CPU
 * path (alaistair76/lxmf-vanity, src/main.rs) and the third-party arithmetic
 * that path calls, none of which is vendored in the reference:
 *   - fiat-crypto 0.3.0 curve25519_64 (5 x 51-bit limbs)     main.rs:44-120
 *   - x25519-dalek 3.0.0 x25519() (RFC 7748 ladder, clamps)  main.rs:194, main.rs:243
 *   - ed25519-dalek 3.0.0 SigningKey -> VerifyingKey (RFC 8032 5.1.5)  main.rs:195
 *   - sha2 0.11.1 Sha256 (FIPS 180-4)                        main.rs:175, main.rs:183-187
 * and the reference's own algorithms:
 *   - step_scalar / previous_scalar / random_start_scalar    main.rs:125-171
 *   - name_hash / lxmf_address / address_of_identity         main.rs:174-197
 *   - Prefix::parse / Prefix::matches                        main.rs:206-224
 *   - prefix_words (big-endian want/mask words)              src/gpu/mod.rs:74-84
 *   - KeyWalk::new / KeyWalk::next_batch (xADD + Montgomery's trick, B=256)
 *                                                            main.rs:242-290
 *   - search (per-key address and prefix test)               main.rs:292-323
 * plus the seeded-input convention of this project (ChaCha20, RFC 8439).
 *
 * Parity pins: the known-answer identity of main.rs:510-525, u(8B), and the
 * walk-vs-plain-X25519 property of main.rs:528-539 (tests/test_oracle.py).
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <pthread.h>
#include <time.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ */
/* GF(2^255-19), 5 x 51-bit unsigned limbs (the fiat-crypto layout).   */

typedef struct { uint64_t v[5]; } fe;
#define M51 ((1ULL << 51) - 1)

static uint64_t ld64(const uint8_t *b) {
    uint64_t x = 0;
    for (int i = 7; i >= 0; i--) x = (x << 8) | b[i];
    return x;
}
static void st64(uint8_t *b, uint64_t x) {
    for (int i = 0; i < 8; i++) { b[i] = (uint8_t)x; x >>= 8; }
}

/* 32 little-endian bytes to limbs, bit 255 ignored (RFC 7748 decodeUCoordinate). */
static fe fe_frombytes(const uint8_t b[32]) {
    uint64_t w0 = ld64(b), w1 = ld64(b + 8), w2 = ld64(b + 16), w3 = ld64(b + 24) & 0x7FFFFFFFFFFFFFFFULL;
    fe h;
    h.v[0] = w0 & M51;
    h.v[1] = ((w0 >> 51) | (w1 << 13)) & M51;
    h.v[2] = ((w1 >> 38) | (w2 << 26)) & M51;
    h.v[3] = ((w2 >> 25) | (w3 << 39)) & M51;
    h.v[4] = (w3 >> 12) & M51;
    return h;
}

static fe fe_carry(fe h) {
    uint64_t c;
    c = h.v[0] >> 51; h.v[0] &= M51; h.v[1] += c;
    c = h.v[1] >> 51; h.v[1] &= M51; h.v[2] += c;
    c = h.v[2] >> 51; h.v[2] &= M51; h.v[3] += c;
    c = h.v[3] >> 51; h.v[3] &= M51; h.v[4] += c;
    c = h.v[4] >> 51; h.v[4] &= M51; h.v[0] += 19 * c;
    c = h.v[0] >> 51; h.v[0] &= M51; h.v[1] += c;
    return h;
}

/* Canonical 32 bytes (value reduced into [0, p)). */
static void fe_tobytes(uint8_t out[32], fe h) {
    h = fe_carry(fe_carry(h));
    /* q = 1 exactly when h >= p. */
    uint64_t q = (h.v[0] + 19) >> 51;
    q = (h.v[1] + q) >> 51;
    q = (h.v[2] + q) >> 51;
    q = (h.v[3] + q) >> 51;
    q = (h.v[4] + q) >> 51;
    h.v[0] += 19 * q;
    uint64_t c;
    c = h.v[0] >> 51; h.v[0] &= M51; h.v[1] += c;
    c = h.v[1] >> 51; h.v[1] &= M51; h.v[2] += c;
    c = h.v[2] >> 51; h.v[2] &= M51; h.v[3] += c;
    c = h.v[3] >> 51; h.v[3] &= M51; h.v[4] += c;
    h.v[4] &= M51;
    st64(out, h.v[0] | (h.v[1] << 51));
    st64(out + 8, (h.v[1] >> 13) | (h.v[2] << 38));
    st64(out + 16, (h.v[2] >> 26) | (h.v[3] << 25));
    st64(out + 24, (h.v[3] >> 39) | (h.v[4] << 12));
}

static fe fe_zero(void) { fe h = {{0, 0, 0, 0, 0}}; return h; }
static fe fe_one(void) { fe h = {{1, 0, 0, 0, 0}}; return h; }
static fe fe_small(uint64_t x) { fe h = {{x, 0, 0, 0, 0}}; return h; }

static fe fe_add(fe f, fe g) {
    fe h;
    for (int i = 0; i < 5; i++) h.v[i] = f.v[i] + g.v[i];
    return fe_carry(h);
}

/* f - g + 4p keeps every limb positive for carried inputs. */
static fe fe_sub(fe f, fe g) {
    fe h;
    h.v[0] = f.v[0] + 0x1FFFFFFFFFFFB4ULL - g.v[0];
    for (int i = 1; i < 5; i++) h.v[i] = f.v[i] + 0x1FFFFFFFFFFFFCULL - g.v[i];
    return fe_carry(h);
}

static fe fe_neg(fe f) { return fe_sub(fe_zero(), f); }

static fe fe_mul(fe f, fe g) {
    const uint64_t *a = f.v, *b = g.v;
    uint64_t b1 = 19 * b[1], b2 = 19 * b[2], b3 = 19 * b[3], b4 = 19 * b[4];
    u128 r0 = (u128)a[0] * b[0] + (u128)a[1] * b4 + (u128)a[2] * b3 + (u128)a[3] * b2 + (u128)a[4] * b1;
    u128 r1 = (u128)a[0] * b[1] + (u128)a[1] * b[0] + (u128)a[2] * b4 + (u128)a[3] * b3 + (u128)a[4] * b2;
    u128 r2 = (u128)a[0] * b[2] + (u128)a[1] * b[1] + (u128)a[2] * b[0] + (u128)a[3] * b4 + (u128)a[4] * b3;
    u128 r3 = (u128)a[0] * b[3] + (u128)a[1] * b[2] + (u128)a[2] * b[1] + (u128)a[3] * b[0] + (u128)a[4] * b4;
    u128 r4 = (u128)a[0] * b[4] + (u128)a[1] * b[3] + (u128)a[2] * b[2] + (u128)a[3] * b[1] + (u128)a[4] * b[0];
    fe h;
    uint64_t c;
    c = (uint64_t)(r0 >> 51); h.v[0] = (uint64_t)r0 & M51; r1 += c;
    c = (uint64_t)(r1 >> 51); h.v[1] = (uint64_t)r1 & M51; r2 += c;
    c = (uint64_t)(r2 >> 51); h.v[2] = (uint64_t)r2 & M51; r3 += c;
    c = (uint64_t)(r3 >> 51); h.v[3] = (uint64_t)r3 & M51; r4 += c;
    c = (uint64_t)(r4 >> 51); h.v[4] = (uint64_t)r4 & M51;
    h.v[0] += 19 * c;
    c = h.v[0] >> 51; h.v[0] &= M51; h.v[1] += c;
    return h;
}

static fe fe_sq(fe f) { return fe_mul(f, f); }

static fe fe_sq_n(fe f, int n) {
    for (int i = 0; i < n; i++) f = fe_sq(f);
    return f;
}

/* z^(p-2): the ref10 addition chain (254 squarings, 11 multiplications),
 * as Fe::invert, main.rs:93-107. */
static fe fe_invert(fe z) {
    fe z2 = fe_sq(z);
    fe z9 = fe_mul(fe_sq_n(z2, 2), z);
    fe z11 = fe_mul(z9, z2);
    fe z2_5_0 = fe_mul(fe_sq(z11), z9);
    fe z2_10_0 = fe_mul(fe_sq_n(z2_5_0, 5), z2_5_0);
    fe z2_20_0 = fe_mul(fe_sq_n(z2_10_0, 10), z2_10_0);
    fe z2_40_0 = fe_mul(fe_sq_n(z2_20_0, 20), z2_20_0);
    fe z2_50_0 = fe_mul(fe_sq_n(z2_40_0, 10), z2_10_0);
    fe z2_100_0 = fe_mul(fe_sq_n(z2_50_0, 50), z2_50_0);
    fe z2_200_0 = fe_mul(fe_sq_n(z2_100_0, 100), z2_100_0);
    fe z2_250_0 = fe_mul(fe_sq_n(z2_200_0, 50), z2_50_0);
    return fe_mul(fe_sq_n(z2_250_0, 5), z11);
}

/* z^((p-5)/8), for square roots (RFC 8032 5.1.3). */
static fe fe_pow22523(fe z) {
    fe z2 = fe_sq(z);
    fe z9 = fe_mul(fe_sq_n(z2, 2), z);
    fe z11 = fe_mul(z9, z2);
    fe z2_5_0 = fe_mul(fe_sq(z11), z9);
    fe z2_10_0 = fe_mul(fe_sq_n(z2_5_0, 5), z2_5_0);
    fe z2_20_0 = fe_mul(fe_sq_n(z2_10_0, 10), z2_10_0);
    fe z2_40_0 = fe_mul(fe_sq_n(z2_20_0, 20), z2_20_0);
    fe z2_50_0 = fe_mul(fe_sq_n(z2_40_0, 10), z2_10_0);
    fe z2_100_0 = fe_mul(fe_sq_n(z2_50_0, 50), z2_50_0);
    fe z2_200_0 = fe_mul(fe_sq_n(z2_100_0, 100), z2_100_0);
    fe z2_250_0 = fe_mul(fe_sq_n(z2_200_0, 50), z2_50_0);
    return fe_mul(fe_sq_n(z2_250_0, 2), z);
}

static int fe_iszero(fe f) {
    uint8_t b[32];
    fe_tobytes(b, f);
    uint8_t acc = 0;
    for (int i = 0; i < 32; i++) acc |= b[i];
    return acc == 0;
}
static int fe_isodd(fe f) {
    uint8_t b[32];
    fe_tobytes(b, f);
    return b[0] & 1;
}
static int fe_eq(fe f, fe g) { return fe_iszero(fe_sub(f, g)); }

/* ------------------------------------------------------------------ */
/* SHA-256 and SHA-512 (FIPS 180-4).                                    */

static const uint32_t K256[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

#define ROR32(x, n) (((x) >> (n)) | ((x) << (32 - (n))))

static void sha256_compress(uint32_t s[8], const uint8_t blk[64]) {
    uint32_t w[64];
    for (int i = 0; i < 16; i++)
        w[i] = (uint32_t)blk[4 * i] << 24 | (uint32_t)blk[4 * i + 1] << 16 | (uint32_t)blk[4 * i + 2] << 8 | blk[4 * i + 3];
    for (int i = 16; i < 64; i++) {
        uint32_t s0 = ROR32(w[i - 15], 7) ^ ROR32(w[i - 15], 18) ^ (w[i - 15] >> 3);
        uint32_t s1 = ROR32(w[i - 2], 17) ^ ROR32(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
    for (int i = 0; i < 64; i++) {
        uint32_t t1 = h + (ROR32(e, 6) ^ ROR32(e, 11) ^ ROR32(e, 25)) + ((e & f) ^ (~e & g)) + K256[i] + w[i];
        uint32_t t2 = (ROR32(a, 2) ^ ROR32(a, 13) ^ ROR32(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
        h = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    s[0] += a; s[1] += b; s[2] += c; s[3] += d; s[4] += e; s[5] += f; s[6] += g; s[7] += h;
}

void orc_sha256(const uint8_t *msg, size_t len, uint8_t out[32]) {
    uint32_t s[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a, 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    size_t off = 0;
    for (; off + 64 <= len; off += 64) sha256_compress(s, msg + off);
    uint8_t blk[128];
    size_t rem = len - off;
    memset(blk, 0, sizeof blk);
    memcpy(blk, msg + off, rem);
    blk[rem] = 0x80;
    size_t nb = (rem + 9 <= 64) ? 64 : 128;
    uint64_t bits = (uint64_t)len * 8;
    for (int i = 0; i < 8; i++) blk[nb - 1 - i] = (uint8_t)(bits >> (8 * i));
    sha256_compress(s, blk);
    if (nb == 128) sha256_compress(s, blk + 64);
    for (int i = 0; i < 8; i++) {
        out[4 * i] = (uint8_t)(s[i] >> 24); out[4 * i + 1] = (uint8_t)(s[i] >> 16);
        out[4 * i + 2] = (uint8_t)(s[i] >> 8); out[4 * i + 3] = (uint8_t)s[i];
    }
}

static const uint64_t K512[80] = {
    0x428a2f98d728ae22ULL, 0x7137449123ef65cdULL, 0xb5c0fbcfec4d3b2fULL, 0xe9b5dba58189dbbcULL,
    0x3956c25bf348b538ULL, 0x59f111f1b605d019ULL, 0x923f82a4af194f9bULL, 0xab1c5ed5da6d8118ULL,
    0xd807aa98a3030242ULL, 0x12835b0145706fbeULL, 0x243185be4ee4b28cULL, 0x550c7dc3d5ffb4e2ULL,
    0x72be5d74f27b896fULL, 0x80deb1fe3b1696b1ULL, 0x9bdc06a725c71235ULL, 0xc19bf174cf692694ULL,
    0xe49b69c19ef14ad2ULL, 0xefbe4786384f25e3ULL, 0x0fc19dc68b8cd5b5ULL, 0x240ca1cc77ac9c65ULL,
    0x2de92c6f592b0275ULL, 0x4a7484aa6ea6e483ULL, 0x5cb0a9dcbd41fbd4ULL, 0x76f988da831153b5ULL,
    0x983e5152ee66dfabULL, 0xa831c66d2db43210ULL, 0xb00327c898fb213fULL, 0xbf597fc7beef0ee4ULL,
    0xc6e00bf33da88fc2ULL, 0xd5a79147930aa725ULL, 0x06ca6351e003826fULL, 0x142929670a0e6e70ULL,
    0x27b70a8546d22ffcULL, 0x2e1b21385c26c926ULL, 0x4d2c6dfc5ac42aedULL, 0x53380d139d95b3dfULL,
    0x650a73548baf63deULL, 0x766a0abb3c77b2a8ULL, 0x81c2c92e47edaee6ULL, 0x92722c851482353bULL,
    0xa2bfe8a14cf10364ULL, 0xa81a664bbc423001ULL, 0xc24b8b70d0f89791ULL, 0xc76c51a30654be30ULL,
    0xd192e819d6ef5218ULL, 0xd69906245565a910ULL, 0xf40e35855771202aULL, 0x106aa07032bbd1b8ULL,
    0x19a4c116b8d2d0c8ULL, 0x1e376c085141ab53ULL, 0x2748774cdf8eeb99ULL, 0x34b0bcb5e19b48a8ULL,
    0x391c0cb3c5c95a63ULL, 0x4ed8aa4ae3418acbULL, 0x5b9cca4f7763e373ULL, 0x682e6ff3d6b2b8a3ULL,
    0x748f82ee5defb2fcULL, 0x78a5636f43172f60ULL, 0x84c87814a1f0ab72ULL, 0x8cc702081a6439ecULL,
    0x90befffa23631e28ULL, 0xa4506cebde82bde9ULL, 0xbef9a3f7b2c67915ULL, 0xc67178f2e372532bULL,
    0xca273eceea26619cULL, 0xd186b8c721c0c207ULL, 0xeada7dd6cde0eb1eULL, 0xf57d4f7fee6ed178ULL,
    0x06f067aa72176fbaULL, 0x0a637dc5a2c898a6ULL, 0x113f9804bef90daeULL, 0x1b710b35131c471bULL,
    0x28db77f523047d84ULL, 0x32caab7b40c72493ULL, 0x3c9ebe0a15c9bebcULL, 0x431d67c49c100d4cULL,
    0x4cc5d4becb3e42b6ULL, 0x597f299cfc657e2aULL, 0x5fcb6fab3ad6faecULL, 0x6c44198c4a475817ULL};

#define ROR64(x, n) (((x) >> (n)) | ((x) << (64 - (n))))

static void sha512_compress(uint64_t s[8], const uint8_t blk[128]) {
    uint64_t w[80];
    for (int i = 0; i < 16; i++) {
        uint64_t x = 0;
        for (int j = 0; j < 8; j++) x = (x << 8) | blk[8 * i + j];
        w[i] = x;
    }
    for (int i = 16; i < 80; i++) {
        uint64_t s0 = ROR64(w[i - 15], 1) ^ ROR64(w[i - 15], 8) ^ (w[i - 15] >> 7);
        uint64_t s1 = ROR64(w[i - 2], 19) ^ ROR64(w[i - 2], 61) ^ (w[i - 2] >> 6);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint64_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
    for (int i = 0; i < 80; i++) {
        uint64_t t1 = h + (ROR64(e, 14) ^ ROR64(e, 18) ^ ROR64(e, 41)) + ((e & f) ^ (~e & g)) + K512[i] + w[i];
        uint64_t t2 = (ROR64(a, 28) ^ ROR64(a, 34) ^ ROR64(a, 39)) + ((a & b) ^ (a & c) ^ (b & c));
        h = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    s[0] += a; s[1] += b; s[2] += c; s[3] += d; s[4] += e; s[5] += f; s[6] += g; s[7] += h;
}

/* SHA-512 of a message shorter than 112 bytes (one block). */
static void sha512_short(const uint8_t *msg, size_t len, uint8_t out[64]) {
    uint64_t s[8] = {0x6a09e667f3bcc908ULL, 0xbb67ae8584caa73bULL, 0x3c6ef372fe94f82bULL, 0xa54ff53a5f1d36f1ULL,
                     0x510e527fade682d1ULL, 0x9b05688c2b3e6c1fULL, 0x1f83d9abfb41bd6bULL, 0x5be0cd19137e2179ULL};
    uint8_t blk[128];
    memset(blk, 0, sizeof blk);
    memcpy(blk, msg, len);
    blk[len] = 0x80;
    uint64_t bits = (uint64_t)len * 8;
    for (int i = 0; i < 8; i++) blk[127 - i] = (uint8_t)(bits >> (8 * i));
    sha512_compress(s, blk);
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) out[8 * i + j] = (uint8_t)(s[i] >> (56 - 8 * j));
}

/* ------------------------------------------------------------------ */
/* X25519 (RFC 7748 section 5).                                        */

static void cswap(fe *a, fe *b, uint64_t bit) {
    uint64_t m = 0 - bit;
    for (int i = 0; i < 5; i++) {
        uint64_t t = m & (a->v[i] ^ b->v[i]);
        a->v[i] ^= t; b->v[i] ^= t;
    }
}

/* x25519(k, u): clamps k as x25519-dalek does, ignores bit 255 of u. */
void orc_x25519(uint8_t out[32], const uint8_t scalar[32], const uint8_t u[32]) {
    uint8_t k[32];
    memcpy(k, scalar, 32);
    k[0] &= 248; k[31] &= 127; k[31] |= 64;
    fe x1 = fe_frombytes(u), x2 = fe_one(), z2 = fe_zero(), x3 = x1, z3 = fe_one();
    const fe a24 = fe_small(121665);
    uint64_t swap = 0;
    for (int t = 254; t >= 0; t--) {
        uint64_t kt = (k[t >> 3] >> (t & 7)) & 1;
        swap ^= kt;
        cswap(&x2, &x3, swap); cswap(&z2, &z3, swap);
        swap = kt;
        fe A = fe_add(x2, z2), AA = fe_sq(A), B = fe_sub(x2, z2), BB = fe_sq(B);
        fe E = fe_sub(AA, BB), C = fe_add(x3, z3), D = fe_sub(x3, z3);
        fe DA = fe_mul(D, A), CB = fe_mul(C, B);
        x3 = fe_sq(fe_add(DA, CB));
        z3 = fe_mul(x1, fe_sq(fe_sub(DA, CB)));
        x2 = fe_mul(AA, BB);
        z2 = fe_mul(E, fe_add(AA, fe_mul(a24, E)));
    }
    cswap(&x2, &x3, swap); cswap(&z2, &z3, swap);
    fe_tobytes(out, fe_mul(x2, fe_invert(z2)));
}

static const uint8_t BASEPOINT9[32] = {9};

void orc_x25519_base(uint8_t out[32], const uint8_t scalar[32]) { orc_x25519(out, scalar, BASEPOINT9); }

/* u(kB) with no clamping: the Montgomery ladder over all 256 bits of k.
 * Used for u(8B) (X25519_BASEPOINT * Scalar::from(8), mod.rs:111, main.rs:244),
 * which no clamped scalar can produce. */
void orc_ladder_unclamped(uint8_t out[32], const uint8_t k[32], const uint8_t u[32]) {
    fe x1 = fe_frombytes(u), x2 = fe_one(), z2 = fe_zero(), x3 = x1, z3 = fe_one();
    const fe a24 = fe_small(121665);
    uint64_t swap = 0;
    for (int t = 255; t >= 0; t--) {
        uint64_t kt = (k[t >> 3] >> (t & 7)) & 1;
        swap ^= kt;
        cswap(&x2, &x3, swap); cswap(&z2, &z3, swap);
        swap = kt;
        fe A = fe_add(x2, z2), AA = fe_sq(A), B = fe_sub(x2, z2), BB = fe_sq(B);
        fe E = fe_sub(AA, BB), C = fe_add(x3, z3), D = fe_sub(x3, z3);
        fe DA = fe_mul(D, A), CB = fe_mul(C, B);
        x3 = fe_sq(fe_add(DA, CB));
        z3 = fe_mul(x1, fe_sq(fe_sub(DA, CB)));
        x2 = fe_mul(AA, BB);
        z2 = fe_mul(E, fe_add(AA, fe_mul(a24, E)));
    }
    cswap(&x2, &x3, swap); cswap(&z2, &z3, swap);
    fe_tobytes(out, fe_mul(x2, fe_invert(z2)));
}

/* ------------------------------------------------------------------ */
/* Ed25519 public key from a 32-byte seed (RFC 8032 5.1.5).             */

typedef struct { fe X, Y, Z, T; } ge;

static fe ED_D, ED_D2, ED_SQRTM1;
static ge ED_B;
static pthread_once_t ed_once = PTHREAD_ONCE_INIT;

static void ed_init(void) {
    /* d = -121665/121666; B = (x, 4/5) with x even. */
    ED_D = fe_mul(fe_neg(fe_small(121665)), fe_invert(fe_small(121666)));
    ED_D2 = fe_add(ED_D, ED_D);
    /* sqrt(-1) = 2^((p-1)/4) */
    {
        /* (p-1)/4 = 2^253 - 5: 2^(2^253 - 5) = (2^(2^250-1))^8 * 2^3 ... use the chain:
         * z^((p-5)/8) with z = 2 gives 2^(2^252-3); then 2^((p-1)/4) = (2^(2^252-3))^2 * 2.  */
        fe t = fe_pow22523(fe_small(2));
        ED_SQRTM1 = fe_mul(fe_sq(t), fe_small(2));
    }
    fe y = fe_mul(fe_small(4), fe_invert(fe_small(5)));
    fe yy = fe_sq(y);
    fe u = fe_sub(yy, fe_one());                 /* y^2 - 1 */
    fe v = fe_add(fe_mul(ED_D, yy), fe_one());   /* d y^2 + 1 */
    /* x = u v^3 (u v^7)^((p-5)/8) */
    fe v3 = fe_mul(fe_sq(v), v);
    fe v7 = fe_mul(fe_sq(v3), v);
    fe x = fe_mul(fe_mul(u, v3), fe_pow22523(fe_mul(u, v7)));
    fe vxx = fe_mul(v, fe_sq(x));
    if (!fe_eq(vxx, u)) x = fe_mul(x, ED_SQRTM1);
    if (fe_isodd(x)) x = fe_neg(x);
    ED_B.X = x; ED_B.Y = y; ED_B.Z = fe_one(); ED_B.T = fe_mul(x, y);
}

/* Unified addition on -x^2 + y^2 = 1 + d x^2 y^2 (extended coordinates). */
static ge ge_add(ge p, ge q) {
    fe A = fe_mul(fe_sub(p.Y, p.X), fe_sub(q.Y, q.X));
    fe B = fe_mul(fe_add(p.Y, p.X), fe_add(q.Y, q.X));
    fe C = fe_mul(fe_mul(p.T, ED_D2), q.T);
    fe D = fe_mul(fe_add(p.Z, p.Z), q.Z);
    fe E = fe_sub(B, A), F = fe_sub(D, C), G = fe_add(D, C), H = fe_add(B, A);
    ge r;
    r.X = fe_mul(E, F); r.Y = fe_mul(G, H); r.T = fe_mul(E, H); r.Z = fe_mul(F, G);
    return r;
}

void orc_ed25519_public(uint8_t pub[32], const uint8_t seed[32]) {
    pthread_once(&ed_once, ed_init);
    uint8_t h[64];
    sha512_short(seed, 32, h);
    h[0] &= 248; h[31] &= 127; h[31] |= 64;
    ge r = {fe_zero(), fe_one(), fe_one(), fe_zero()};
    for (int t = 254; t >= 0; t--) {
        r = ge_add(r, r);
        if ((h[t >> 3] >> (t & 7)) & 1) r = ge_add(r, ED_B);
    }
    fe zi = fe_invert(r.Z);
    fe x = fe_mul(r.X, zi), y = fe_mul(r.Y, zi);
    fe_tobytes(pub, y);
    pub[31] |= (uint8_t)(fe_isodd(x) << 7);
}

/* ------------------------------------------------------------------ */
/* Scalars (main.rs:125-171) and seeded draws (ChaCha20, RFC 8439).      */

/* k + 8n, little-endian 256-bit (main.rs:125-137). */
void orc_step_scalar(uint8_t out[32], const uint8_t k[32], uint64_t n) {
    u128 carry = (u128)n * 8;
    for (int i = 0; i < 32; i++) {
        u128 sum = (u128)k[i] + (carry & 0xFF);
        out[i] = (uint8_t)sum;
        carry = (carry >> 8) + (sum >> 8);
    }
}

/* k - 8 (main.rs:140-152). */
void orc_previous_scalar(uint8_t out[32], const uint8_t k[32]) {
    int borrow = 8;
    for (int i = 0; i < 32; i++) {
        int v = (int)k[i] - borrow;
        out[i] = (uint8_t)(v & 0xFF);
        borrow = v < 0 ? 1 : 0;
    }
}

/* The clamping and rejection rule of random_start_scalar (main.rs:157-171):
 * returns 1 and clamps `k` in place when it is acceptable. */
int orc_clamp_start(uint8_t k[32]) {
    k[0] &= 248; k[31] &= 127; k[31] |= 64;
    int high_all_set = k[31] == 127, low_all_clear = k[31] == 64;
    for (int i = 9; i < 31; i++) high_all_set &= k[i] == 0xFF;
    for (int i = 0; i < 31; i++) low_all_clear &= k[i] == 0;
    return !high_all_set && !low_all_clear;
}

static void chacha20_block(uint8_t out[64], const uint32_t key[8], uint32_t counter) {
    uint32_t s[16] = {0x61707865, 0x3320646e, 0x79622d32, 0x6b206574,
                      key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                      counter, 0, 0, 0};
    uint32_t x[16];
    memcpy(x, s, sizeof x);
#define QR(a, b, c, d) \
    x[a] += x[b]; x[d] ^= x[a]; x[d] = (x[d] << 16) | (x[d] >> 16); \
    x[c] += x[d]; x[b] ^= x[c]; x[b] = (x[b] << 12) | (x[b] >> 20); \
    x[a] += x[b]; x[d] ^= x[a]; x[d] = (x[d] << 8) | (x[d] >> 24);  \
    x[c] += x[d]; x[b] ^= x[c]; x[b] = (x[b] << 7) | (x[b] >> 25);
    for (int i = 0; i < 10; i++) {
        QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
        QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
    }
#undef QR
    for (int i = 0; i < 16; i++) {
        uint32_t v = x[i] + s[i];
        out[4 * i] = (uint8_t)v; out[4 * i + 1] = (uint8_t)(v >> 8);
        out[4 * i + 2] = (uint8_t)(v >> 16); out[4 * i + 3] = (uint8_t)(v >> 24);
    }
}

/* `len` bytes of the keystream for `seed`, starting at byte `offset`.
 * Key = seed as a u64 little-endian in bytes 0-7, zeros elsewhere; nonce 0;
 * block counter from 0. */
void orc_chacha20_stream(uint64_t seed, uint64_t offset, uint8_t *out, size_t len) {
    uint32_t key[8] = {(uint32_t)seed, (uint32_t)(seed >> 32), 0, 0, 0, 0, 0, 0};
    uint8_t blk[64];
    while (len > 0) {
        uint32_t ctr = (uint32_t)(offset / 64);
        size_t skip = offset % 64, take = 64 - skip;
        if (take > len) take = len;
        chacha20_block(blk, key, ctr);
        memcpy(out, blk + skip, take);
        out += take; len -= take; offset += take;
    }
}

/* The seeded identity and walker scalars: scalar 0 and the Ed25519 seed are
 * the first 64 bytes; every further walker draws the next 32 bytes.  A
 * rejected draw (orc_clamp_start) is replaced by the next 32 bytes.
 * Returns the stream offset after the draws. */
uint64_t orc_seeded_identity(uint64_t seed, uint8_t scalar0[32], uint8_t ed_seed[32], uint64_t *offset_out) {
    uint64_t off = 0;
    for (;;) {
        orc_chacha20_stream(seed, off, scalar0, 32);
        off += 32;
        if (orc_clamp_start(scalar0)) break;
    }
    orc_chacha20_stream(seed, off, ed_seed, 32);
    off += 32;
    if (offset_out) *offset_out = off;
    return off;
}

/* `count` further walker scalars from stream offset `offset`. */
uint64_t orc_seeded_scalars(uint64_t seed, uint64_t offset, uint8_t *scalars, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) {
        for (;;) {
            orc_chacha20_stream(seed, offset, scalars + 32 * i, 32);
            offset += 32;
            if (orc_clamp_start(scalars + 32 * i)) break;
        }
    }
    return offset;
}

/* ------------------------------------------------------------------ */
/* Addresses and prefixes (main.rs:174-224, mod.rs:74-84).              */

void orc_name_hash(const uint8_t *aspect, size_t len, uint8_t out[10]) {
    uint8_t h[32];
    orc_sha256(aspect, len, h);
    memcpy(out, h, 10);
}

void orc_lxmf_address(const uint8_t name_hash[10], const uint8_t x_pub[32], const uint8_t ed_pub[32], uint8_t out[16]) {
    uint8_t pk[64], ih[32], mat[26], h[32];
    memcpy(pk, x_pub, 32);
    memcpy(pk + 32, ed_pub, 32);
    orc_sha256(pk, 64, ih);
    memcpy(mat, name_hash, 10);
    memcpy(mat + 10, ih, 16);
    orc_sha256(mat, 26, h);
    memcpy(out, h, 16);
}

void orc_address_of_identity(const uint8_t identity[64], const uint8_t name_hash[10], uint8_t out[16]) {
    uint8_t x_pub[32], ed_pub[32];
    orc_x25519_base(x_pub, identity);
    orc_ed25519_public(ed_pub, identity + 32);
    orc_lxmf_address(name_hash, x_pub, ed_pub, out);
}

/* Prefix::parse: 1..32 hex digits, any case; odd lengths padded with '0'.
 * Returns the nibble count, or -1 when the text is not a prefix. */
int orc_prefix_parse(const char *s, uint8_t bytes[16]) {
    size_t n = strlen(s);
    if (n == 0 || n > 32) return -1;
    memset(bytes, 0, 16);
    for (size_t i = 0; i < n; i++) {
        int c = s[i], v;
        if (c >= '0' && c <= '9') v = c - '0';
        else if (c >= 'a' && c <= 'f') v = c - 'a' + 10;
        else if (c >= 'A' && c <= 'F') v = c - 'A' + 10;
        else return -1;
        bytes[i / 2] |= (uint8_t)(v << ((i % 2 == 0) ? 4 : 0));
    }
    return (int)n;
}

int orc_prefix_matches(const uint8_t bytes[16], int nibbles, const uint8_t address[16]) {
    int whole = nibbles / 2;
    if (memcmp(address, bytes, (size_t)whole) != 0) return 0;
    return nibbles % 2 == 0 || (address[whole] >> 4) == (bytes[whole] >> 4);
}

/* Big-endian want/mask words of the address bytes the prefix fixes. */
void orc_prefix_words(const uint8_t bytes[16], int nibbles, uint32_t want[4], uint32_t mask[4]) {
    uint8_t w[16] = {0}, m[16] = {0};
    for (int i = 0; i < nibbles; i++) {
        int shift = (i % 2 == 0) ? 4 : 0;
        m[i / 2] |= (uint8_t)(0xF << shift);
        w[i / 2] |= (uint8_t)(((bytes[i / 2] >> shift) & 0xF) << shift);
    }
    for (int k = 0; k < 4; k++) {
        want[k] = (uint32_t)w[4 * k] << 24 | (uint32_t)w[4 * k + 1] << 16 | (uint32_t)w[4 * k + 2] << 8 | w[4 * k + 3];
        mask[k] = (uint32_t)m[4 * k] << 24 | (uint32_t)m[4 * k + 1] << 16 | (uint32_t)m[4 * k + 2] << 8 | m[4 * k + 3];
    }
}

/* ------------------------------------------------------------------ */
/* The key walk (KeyWalk, main.rs:230-290) and the search (main.rs:292-323). */

#define WALK_BATCH 256

typedef struct {
    uint8_t start[32];
    uint64_t next_n;
    fe xp, zp, xc, zc;
    fe q_plus, q_minus;
} keywalk;

static fe U8B;
static pthread_once_t u8b_once = PTHREAD_ONCE_INIT;
static void u8b_init(void) {
    uint8_t k[32] = {8}, u[32];
    orc_ladder_unclamped(u, k, BASEPOINT9);
    U8B = fe_frombytes(u);
}

void orc_u8b(uint8_t out[32]) {
    pthread_once(&u8b_once, u8b_init);
    fe_tobytes(out, U8B);
}

static void keywalk_new(keywalk *w, const uint8_t start[32]) {
    pthread_once(&u8b_once, u8b_init);
    uint8_t prev[32], u[32];
    memcpy(w->start, start, 32);
    w->next_n = 0;
    orc_previous_scalar(prev, start);
    orc_x25519_base(u, prev);
    w->xp = fe_frombytes(u); w->zp = fe_one();
    orc_x25519_base(u, start);
    w->xc = fe_frombytes(u); w->zc = fe_one();
    w->q_plus = fe_add(U8B, fe_one());
    w->q_minus = fe_sub(U8B, fe_one());
}

/* The next `len` (<= WALK_BATCH) public keys; returns the n of the first. */
static uint64_t keywalk_next_batch(keywalk *w, uint8_t (*out)[32], int len) {
    uint64_t first = w->next_n;
    fe xs[WALK_BATCH], zs[WALK_BATCH], prefix[WALK_BATCH];
    for (int i = 0; i < len; i++) {
        xs[i] = w->xc; zs[i] = w->zc;
        /* xADD: P(n+1) = P(n) + Q with P(n) - Q = P(n-1), Q = 8B affine. */
        fe t1 = fe_mul(fe_sub(w->xc, w->zc), w->q_plus);
        fe t2 = fe_mul(fe_add(w->xc, w->zc), w->q_minus);
        fe xn = fe_mul(w->zp, fe_sq(fe_add(t1, t2)));
        fe zn = fe_mul(w->xp, fe_sq(fe_sub(t1, t2)));
        w->xp = w->xc; w->zp = w->zc; w->xc = xn; w->zc = zn;
    }
    fe acc = fe_one();
    for (int i = 0; i < len; i++) { prefix[i] = acc; acc = fe_mul(acc, zs[i]); }
    fe inv = fe_invert(acc);
    for (int i = len - 1; i >= 0; i--) {
        fe z_inv = fe_mul(inv, prefix[i]);
        inv = fe_mul(inv, zs[i]);
        fe_tobytes(out[i], fe_mul(xs[i], z_inv));
    }
    w->next_n += (uint64_t)len;
    return first;
}

/* Public keys u(start + 8n) for n in [0, count), by the walk. */
void orc_walk_keys(const uint8_t start[32], uint64_t count, uint8_t *out) {
    keywalk w;
    keywalk_new(&w, start);
    uint8_t (*keys)[32] = (uint8_t (*)[32])out;
    while (w.next_n < count) {
        uint64_t left = count - w.next_n;
        int len = left < WALK_BATCH ? (int)left : WALK_BATCH;
        keywalk_next_batch(&w, keys + w.next_n, len);
    }
}

/* The search of one walker over walk indices [0, count): records every index
 * whose address matches the prefix (up to max_hits; the return value is the
 * full count) and the addresses of the first `dump` indices. */
uint64_t orc_search_window(const uint8_t start[32], const uint8_t ed_pub[32], const uint8_t name_hash[10],
                           const uint8_t prefix_bytes[16], int nibbles, uint64_t count,
                           uint64_t *hits, uint64_t max_hits, uint8_t *dump_addr, uint64_t dump) {
    keywalk w;
    keywalk_new(&w, start);
    uint8_t keys[WALK_BATCH][32], addr[16];
    uint64_t found = 0;
    while (w.next_n < count) {
        uint64_t left = count - w.next_n;
        int len = left < WALK_BATCH ? (int)left : WALK_BATCH;
        uint64_t first = keywalk_next_batch(&w, keys, len);
        for (int i = 0; i < len; i++) {
            uint64_t n = first + (uint64_t)i;
            orc_lxmf_address(name_hash, keys[i], ed_pub, addr);
            if (n < dump) memcpy(dump_addr + 16 * n, addr, 16);
            if (orc_prefix_matches(prefix_bytes, nibbles, addr)) {
                if (found < max_hits) hits[found] = n;
                found++;
            }
        }
    }
    return found;
}

/* ------------------------------------------------------------------ */
/* Field primitives on 8 little-endian words (the microbench interface).
 * Inputs drop bit 255 (as fe_from_words does, common.h:131-142); outputs are
 * canonical. op: 0 mul, 1 square, 2 invert. */

static fe fe_fromwords(const uint32_t w[8]) {
    uint8_t b[32];
    for (int i = 0; i < 8; i++) { b[4 * i] = (uint8_t)w[i]; b[4 * i + 1] = (uint8_t)(w[i] >> 8);
                                  b[4 * i + 2] = (uint8_t)(w[i] >> 16); b[4 * i + 3] = (uint8_t)(w[i] >> 24); }
    return fe_frombytes(b);
}
static void fe_towords(uint32_t w[8], fe f) {
    uint8_t b[32];
    fe_tobytes(b, f);
    for (int i = 0; i < 8; i++)
        w[i] = (uint32_t)b[4 * i] | (uint32_t)b[4 * i + 1] << 8 | (uint32_t)b[4 * i + 2] << 16 | (uint32_t)b[4 * i + 3] << 24;
}

void orc_fe_op(int op, const uint32_t *a, const uint32_t *b, uint32_t *out, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) {
        fe x = fe_fromwords(a + 8 * i), r;
        if (op == 0) r = fe_mul(x, fe_fromwords(b + 8 * i));
        else if (op == 1) r = fe_sq(x);
        else r = fe_invert(x);
        fe_towords(out + 8 * i, r);
    }
}

/* Batch inversion by Montgomery's trick over groups of `group` elements
 * (the walk's structure, main.rs:274-287): a zero anywhere in a group
 * zeroes the whole group, as in the walk. */
void orc_fe_batch_invert(const uint32_t *a, uint32_t *out, uint64_t count, int group) {
    fe prefix[256], zs[256];
    for (uint64_t g0 = 0; g0 < count; g0 += (uint64_t)group) {
        int len = (int)((count - g0) < (uint64_t)group ? (count - g0) : (uint64_t)group);
        fe acc = fe_one();
        for (int i = 0; i < len; i++) { zs[i] = fe_fromwords(a + 8 * (g0 + i)); prefix[i] = acc; acc = fe_mul(acc, zs[i]); }
        fe inv = fe_invert(acc);
        for (int i = len - 1; i >= 0; i--) {
            fe_towords(out + 8 * (g0 + i), fe_mul(inv, prefix[i]));
            inv = fe_mul(inv, zs[i]);
        }
    }
}

/* The address chain on whole 64-byte public keys: out = first 16 bytes of
 * SHA-256(name_hash || SHA-256(pk)[0..16]). */
void orc_address_chain(const uint8_t *pks, const uint8_t name_hash[10], uint8_t *out, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) orc_lxmf_address(name_hash, pks + 64 * i, pks + 64 * i + 32, out + 16 * i);
}

/* ------------------------------------------------------------------ */
/* Timed CPU search: `threads` threads, each walking its own start for
 * `keys_per_thread` keys (rounded up to whole batches) with the search's
 * per-key address and prefix test.  Returns keys per second (wall clock). */

typedef struct {
    uint8_t start[32], ed_pub[32], nh[10], pfx[16];
    int nibbles;
    uint64_t keys, hits;
} bench_job;

static void *bench_thread(void *arg) {
    bench_job *j = (bench_job *)arg;
    keywalk w;
    keywalk_new(&w, j->start);
    uint8_t keys[WALK_BATCH][32], addr[16];
    uint64_t hits = 0;
    while (w.next_n < j->keys) {
        keywalk_next_batch(&w, keys, WALK_BATCH);
        for (int i = 0; i < WALK_BATCH; i++) {
            orc_lxmf_address(j->nh, keys[i], j->ed_pub, addr);
            hits += (uint64_t)orc_prefix_matches(j->pfx, j->nibbles, addr);
        }
    }
    j->hits = hits;
    j->keys = w.next_n;
    return NULL;
}

double orc_bench_search(int threads, uint64_t keys_per_thread, uint64_t seed, const uint8_t prefix_bytes[16], int nibbles,
                        uint64_t *keys_done, uint64_t *hits_out) {
    if (threads < 1) threads = 1;
    bench_job *jobs = (bench_job *)calloc((size_t)threads, sizeof(bench_job));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    uint8_t scalar0[32], ed_seed[32], ed_pub[32], nh[10];
    uint64_t off;
    orc_seeded_identity(seed, scalar0, ed_seed, &off);
    orc_ed25519_public(ed_pub, ed_seed);
    orc_name_hash((const uint8_t *)"lxmf.delivery", 13, nh);
    pthread_once(&u8b_once, u8b_init);
    for (int t = 0; t < threads; t++) {
        if (t == 0) memcpy(jobs[t].start, scalar0, 32);
        else off = orc_seeded_scalars(seed, off, jobs[t].start, 1);
        memcpy(jobs[t].ed_pub, ed_pub, 32);
        memcpy(jobs[t].nh, nh, 10);
        memcpy(jobs[t].pfx, prefix_bytes, 16);
        jobs[t].nibbles = nibbles;
        jobs[t].keys = keys_per_thread;
    }
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (int t = 0; t < threads; t++) pthread_create(&tid[t], NULL, bench_thread, &jobs[t]);
    uint64_t total = 0, hits = 0;
    for (int t = 0; t < threads; t++) { pthread_join(tid[t], NULL); total += jobs[t].keys; hits += jobs[t].hits; }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    double secs = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    if (keys_done) *keys_done = total;
    if (hits_out) *hits_out = hits;
    free(jobs); free(tid);
    return secs > 0 ? (double)total / secs : 0.0;
}
