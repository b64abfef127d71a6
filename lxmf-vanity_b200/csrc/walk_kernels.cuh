// The key-walk search kernels (sm_100a): shared pieces and the x-only walk.
//
// Replaces the reference's init_walk / walk (src/gpu/kernel.cu:21-36) and
// their body init_thread / walk_thread (src/gpu/common.h:261-365).
//
// Each lane walks X25519 private keys k, k+8, k+16, ... (walk index n is key
// k + 8n).  Two walks produce the same keys (so the same hashes and hits):
//
// x-only walk (walk_kernel, the reference's algorithm).  Lane state in HBM is
// the projective pair P(n-1) = (Xp:Zp), P(n) = (Xc:Zc), 4 x 32 bytes,
// word-major (state[w * lanes + lane]) so that every access is coalesced.
// One launch walks `iters` batches of B keys per lane:
//   1. B steps of the differential addition P(n+1) = P(n) + Q, Q = 8B affine:
//      X' = Zp (q Xc - Zc)^2, Z' = Xp (Xc - q Zc)^2 (4M + 2S; the reference's
//      form, common.h:316-325, differs by a factor 4 that projective
//      coordinates ignore).  Each key's Zc and Y = Xc * (Z0...Zi-1) go to the
//      lane's local batch buffer;
//   2. one inversion of Z0 * ... * Z(B-1) (Montgomery's trick);
//   3. backwards over the batch: u = Y * inv, inv *= Zi (2M per key); u is
//      canonicalised, hashed to its destination hash and compared with the
//      prefix; a match takes a slot of the hit queue by atomicAdd.
// Per key: 8M + 2S, plus 1/B of an inversion, one canonicalisation and three
// SHA-256 compressions: the reference's work per key.
//
// The grouped walk (group_kernels.cuh) reaches the same keys with affine
// additions around a centre point and about half the field work.
#pragma once
#include <cstdint>

#include "fe25519.cuh"
#include "sha256_lxmf.cuh"

namespace lxk {

struct Hit {
    uint32_t thread;
    uint32_t reserved;
    uint64_t n;
};

// What a finished key is checked against and where results go.
struct EmitArgs {
    lxsha::AddrConsts ac;
    uint32_t* hit_count;
    Hit* hits;
    uint32_t max_hits;
    uint32_t dump_lanes;
    uint32_t dump_keys;
    uint32_t* dump_u;     // [dump_lanes][dump_keys][8], or null
    uint32_t* dump_addr;  // [dump_lanes][dump_keys][4], or null
};

struct WalkArgs {
    uint32_t* state;    // [32][lanes]: Xp, Zp, Xc, Zc, 8 words each
    uint64_t* ns;       // [lanes]: walk index of P(n) = (Xc:Zc)
    uint32_t lanes;
    uint32_t iters;
    fe q;               // u(8B)
    EmitArgs em;
};

__device__ __forceinline__ fe load_fe(const uint32_t* st, int e, uint32_t lane, uint32_t lanes) {
    fe r;
#pragma unroll
    for (int w = 0; w < 8; w++) r.v[w] = st[(size_t)(e * 8 + w) * lanes + lane];
    return r;
}

__device__ __forceinline__ void store_fe(uint32_t* st, int e, uint32_t lane, uint32_t lanes, const fe& x) {
#pragma unroll
    for (int w = 0; w < 8; w++) st[(size_t)(e * 8 + w) * lanes + lane] = x.v[w];
}

// u(key) is final and canonical: hash, compare, record.  key0 is the lane's
// first walk index in this launch (the dump window starts there).  DUMP: the
// kernel was launched with a dump window; launches without one run kernels
// built without the dump code (the per-key test and stores cost 0.7%).
template <bool DUMP>
__device__ __forceinline__ void emit_key(const EmitArgs& a, uint32_t lane, uint64_t key, uint64_t key0, const fe& u) {
    uint32_t d[4];
    lxsha::dest_hash(u.v, a.ac.ed, a.ac, d);
    const bool match = ((d[0] & a.ac.mask[0]) == a.ac.want[0]) & ((d[1] & a.ac.mask[1]) == a.ac.want[1]) &
                       ((d[2] & a.ac.mask[2]) == a.ac.want[2]) & ((d[3] & a.ac.mask[3]) == a.ac.want[3]);
    if (match) {
        const uint32_t slot = atomicAdd(a.hit_count, 1u);
        if (slot < a.max_hits) {
            a.hits[slot].thread = lane;
            a.hits[slot].reserved = 0;
            a.hits[slot].n = key;
        }
    }
    if (DUMP && lane < a.dump_lanes) {
        const uint64_t m = key - key0;
        if (m < a.dump_keys) {
            const size_t at = (size_t)lane * a.dump_keys + m;
            if (a.dump_u) {
#pragma unroll
                for (int w = 0; w < 8; w++) a.dump_u[at * 8 + w] = u.v[w];
            }
            if (a.dump_addr) {
#pragma unroll
                for (int w = 0; w < 4; w++) a.dump_addr[at * 4 + w] = d[w];
            }
        }
    }
}

// SYNC: a block barrier after each batch keeps the block's warps in the same
// phase (see group_walk_kernel); threads past the last lane then walk a copy
// of the last lane and neither emit nor store.
template <int B, int BLOCK, int MINB, bool SYNC, bool DUMP>
static __global__ void __launch_bounds__(BLOCK, MINB) walk_kernel(const __grid_constant__ WalkArgs a) {
    const uint32_t tid = blockIdx.x * BLOCK + threadIdx.x;
    if (!SYNC && tid >= a.lanes) return;
    const bool active = tid < a.lanes;
    const uint32_t lane = active ? tid : a.lanes - 1;
    fe xp = load_fe(a.state, 0, lane, a.lanes);
    fe zp = load_fe(a.state, 1, lane, a.lanes);
    fe xc = load_fe(a.state, 2, lane, a.lanes);
    fe zc = load_fe(a.state, 3, lane, a.lanes);
    const uint64_t key0 = a.ns[lane];
    uint64_t n = key0;
    fe ys[B], zs[B];

#pragma unroll 1
    for (uint32_t it = 0; it < a.iters; ++it) {
        fe acc = fe_one();
#pragma unroll 1
        for (int i = 0; i < B; ++i) {
            ys[i] = fe_mul(xc, acc);
            zs[i] = zc;
            acc = fe_mul(acc, zc);
            const fe t1 = fe_sub(fe_mul(xc, a.q), zc);
            const fe t2 = fe_sub(xc, fe_mul(zc, a.q));
            const fe xn = fe_mul(zp, fe_sqr(t1));
            const fe zn = fe_mul(xp, fe_sqr(t2));
            xp = xc;
            zp = zc;
            xc = xn;
            zc = zn;
        }
        fe inv = fe_invert(acc);
#pragma unroll 1
        for (int i = B - 1; i >= 0; --i) {
            const fe u = fe_canon(fe_mul(ys[i], inv));
            inv = fe_mul(inv, zs[i]);
            if (active) emit_key<DUMP>(a.em, lane, n + (uint64_t)i, key0, u);
        }
        n += B;
        if (SYNC) __syncthreads();
    }

    if (active) {
        store_fe(a.state, 0, lane, a.lanes, xp);
        store_fe(a.state, 1, lane, a.lanes, zp);
        store_fe(a.state, 2, lane, a.lanes, xc);
        store_fe(a.state, 3, lane, a.lanes, zc);
        a.ns[lane] = n;
    }
}

// Backend::init (mod.rs:48): lane t from u(k-8), u(k) as 16 LE words, Z = 1.
// Bit 255 of each u is dropped, as fe_from_words does (common.h:131-142).
static __global__ void init_kernel(uint32_t* state, uint64_t* ns, const uint32_t* __restrict__ upc, uint32_t lanes) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= lanes) return;
    fe xp, xc;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        xp.v[w] = upc[(size_t)lane * 16 + w];
        xc.v[w] = upc[(size_t)lane * 16 + 8 + w];
    }
    xp.v[7] &= 0x7fffffffu;
    xc.v[7] &= 0x7fffffffu;
    store_fe(state, 0, lane, lanes, xp);
    store_fe(state, 1, lane, lanes, fe_one());
    store_fe(state, 2, lane, lanes, xc);
    store_fe(state, 3, lane, lanes, fe_one());
    ns[lane] = 0;
}

// ---- Scalar multiples of Q = 8B on the GPU.

// The Montgomery ladder (RFC 7748's step, a24 = 121665, swaps by masks: no
// branch on a secret bit) over bits [nbits-1, 0] of the 256-bit scalar s
// (8 LE words), base point u = q: ends with (X2:Z2) = s Q, (X3:Z3) = (s+1) Q.
__device__ __forceinline__ void ladder(const uint32_t s[8], int nbits, const fe& q, fe& x2, fe& z2, fe& x3, fe& z3) {
    x2 = fe_one();
    z2 = fe_zero();
    x3 = q;
    z3 = fe_one();
    uint32_t swap = 0;
#pragma unroll 1
    for (int t = nbits - 1; t >= 0; --t) {
        const uint32_t bit = (s[t >> 5] >> (t & 31)) & 1u;
        swap ^= bit;
        fe_cswap(x2, x3, 0u - swap);
        fe_cswap(z2, z3, 0u - swap);
        swap = bit;
        const fe A = fe_add(x2, z2), AA = fe_sqr(A);
        const fe Bv = fe_sub(x2, z2), BB = fe_sqr(Bv);
        const fe E = fe_sub(AA, BB);
        const fe C = fe_add(x3, z3), D = fe_sub(x3, z3);
        const fe DA = fe_mul(D, A), CB = fe_mul(C, Bv);
        x3 = fe_sqr(fe_add(DA, CB));
        z3 = fe_mul(q, fe_sqr(fe_sub(DA, CB)));
        x2 = fe_mul(AA, BB);
        z2 = fe_mul(E, fe_add(AA, fe_mul_small(E, 121665u)));
    }
    fe_cswap(x2, x3, 0u - swap);
    fe_cswap(z2, z3, 0u - swap);
}

// Lane `lane`'s start scalar k (8 LE words) as k/8 + add (add may be -1):
// the multiple of Q that is key k + 8 add.
__device__ __forceinline__ void scalar_over_8(const uint32_t* __restrict__ scalars, uint32_t lane, int add,
                                              uint32_t s[8]) {
    uint32_t k[8];
#pragma unroll
    for (int w = 0; w < 8; w++) k[w] = scalars[(size_t)lane * 8 + w];
#pragma unroll
    for (int w = 0; w < 7; w++) s[w] = __funnelshift_r(k[w], k[w + 1], 3);
    s[7] = k[7] >> 3;
    // s += add, as a 256-bit two's-complement addition
    uint32_t carry = 0;
    const uint32_t ext = add < 0 ? 0xffffffffu : 0u;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        const uint64_t t = (uint64_t)s[w] + (w == 0 ? (uint32_t)add : ext) + carry;
        s[w] = (uint32_t)t;
        carry = (uint32_t)(t >> 32);
    }
}

// x-only start: (P(-1), P(0)) = ((k-8)B, kB), left projective (replacing the
// CPU start points of first_public_keys, mod.rs:212-228, for the walk).
static __global__ void __launch_bounds__(128) ladder_kernel(uint32_t* state, uint64_t* ns, const uint32_t* __restrict__ scalars,
                                                     uint32_t lanes, fe q) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= lanes) return;
    uint32_t s[8];
    scalar_over_8(scalars, lane, -1, s);
    fe x2, z2, x3, z3;
    ladder(s, 252, q, x2, z2, x3, z3);
    store_fe(state, 0, lane, lanes, x2);
    store_fe(state, 1, lane, lanes, z2);
    store_fe(state, 2, lane, lanes, x3);
    store_fe(state, 3, lane, lanes, z3);
    ns[lane] = 0;
}

// first_public_keys (mod.rs:212-228) on the GPU: u(k-8) and u(k) as 16
// canonical little-endian words per lane, the input of Backend::init.  One
// inversion of Z2 * Z3 serves both coordinates.
static __global__ void __launch_bounds__(128) first_keys_kernel(uint32_t* __restrict__ upc, const uint32_t* __restrict__ scalars,
                                                         uint32_t lanes, fe q) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= lanes) return;
    uint32_t s[8];
    scalar_over_8(scalars, lane, -1, s);
    fe x2, z2, x3, z3;
    ladder(s, 252, q, x2, z2, x3, z3);
    const fe inv = fe_invert(fe_mul(z2, z3));
    const fe u_prev = fe_canon(fe_mul(x2, fe_mul(inv, z3)));
    const fe u_cur = fe_canon(fe_mul(x3, fe_mul(inv, z2)));
#pragma unroll
    for (int w = 0; w < 8; w++) {
        upc[(size_t)lane * 16 + w] = u_prev.v[w];
        upc[(size_t)lane * 16 + 8 + w] = u_cur.v[w];
    }
}

}  // namespace lxk
