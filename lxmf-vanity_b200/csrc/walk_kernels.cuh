// The key-walk search kernels (sm_100a).
//
// Replaces the reference's init_walk / walk (src/gpu/kernel.cu:21-36) and
// their body init_thread / walk_thread (src/gpu/common.h:261-365).
//
// Each lane walks X25519 private keys k, k+8, k+16, ... .  Its state in HBM
// is the projective pair P(n-1) = (Xp:Zp), P(n) = (Xc:Zc), 4 x 32 bytes, kept
// structure-of-arrays (word-major: state[w * lanes + lane]) so that every
// load and store of the state is coalesced.  One launch walks `iters`
// batches of B keys per lane:
//   1. B steps of the x-only differential addition P(n+1) = P(n) + Q, Q = 8B
//      affine: X' = Zp (q Xc - Zc)^2, Z' = Xp (Xc - q Zc)^2 (4M + 2S; the
//      reference's form, common.h:316-325, differs by the factor 4 that
//      projective coordinates ignore).  Each key's Zc and Y = Xc * (Z0..Zi-1)
//      go to the lane's local batch buffer;
//   2. one inversion of Z0 * ... * Z(B-1) (Montgomery's trick);
//   3. backwards over the batch: u = Y * inv, inv *= Zi (2M per key); u is
//      canonicalised, hashed to its destination hash and compared with the
//      prefix; a match takes a slot of the hit queue by atomicAdd.
// Per key: 8M + 2S, plus 1/B of an inversion, one canonicalisation and three
// SHA-256 compressions (the same work as the reference per key).
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

struct WalkArgs {
    uint32_t* state;    // [32][lanes]: Xp, Zp, Xc, Zc, 8 words each
    uint64_t* ns;       // [lanes]: walk index of P(n) = (Xc:Zc)
    uint32_t lanes;
    uint32_t iters;
    fe q;               // u(8B)
    lxsha::AddrConsts ac;
    uint32_t* hit_count;
    Hit* hits;
    uint32_t max_hits;
    uint32_t dump_lanes;
    uint32_t dump_keys;
    uint32_t* dump_u;     // [dump_lanes][dump_keys][8], or null
    uint32_t* dump_addr;  // [dump_lanes][dump_keys][4], or null
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

// u(key) is final and canonical: hash, compare, record.
__device__ __forceinline__ void emit_key(const WalkArgs& a, uint32_t lane, uint64_t key, uint64_t key0, const fe& u) {
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
    if (lane < a.dump_lanes) {
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

template <int B, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) walk_kernel(const __grid_constant__ WalkArgs a) {
    const uint32_t lane = blockIdx.x * BLOCK + threadIdx.x;
    if (lane >= a.lanes) return;
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
            emit_key(a, lane, n + (uint64_t)i, key0, u);
        }
        n += B;
    }

    store_fe(a.state, 0, lane, a.lanes, xp);
    store_fe(a.state, 1, lane, a.lanes, zp);
    store_fe(a.state, 2, lane, a.lanes, xc);
    store_fe(a.state, 3, lane, a.lanes, zc);
    a.ns[lane] = n;
}

// Backend::init (mod.rs:48): lane t from u(k-8), u(k) as 16 LE words, Z = 1.
// Bit 255 of each u is dropped, as fe_from_words does (common.h:131-142).
__global__ void init_kernel(uint32_t* state, uint64_t* ns, const uint32_t* __restrict__ upc, uint32_t lanes) {
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

// Start points on the GPU (replacing first_public_keys, mod.rs:212-228): for
// a start scalar k (a multiple of 8), the Montgomery ladder over s = k/8 - 1
// with base point Q = 8B ends with (X2:Z2) = s Q = (k-8) B and
// (X3:Z3) = (s+1) Q = k B: exactly the walk's (P(n-1), P(n)) at n = 0, left
// projective.  The ladder step is RFC 7748's, with a24 = 121665 and swaps by
// masks (no branch on a secret bit).
__device__ __forceinline__ void ladder_pair(const uint32_t* __restrict__ scalars, uint32_t lane, const fe& q, fe& x2,
                                            fe& z2, fe& x3, fe& z3) {
    uint32_t k[8], s[8];
#pragma unroll
    for (int w = 0; w < 8; w++) k[w] = scalars[(size_t)lane * 8 + w];
#pragma unroll
    for (int w = 0; w < 7; w++) s[w] = __funnelshift_r(k[w], k[w + 1], 3);
    s[7] = k[7] >> 3;
    // s -= 1
    uint32_t borrow = 1;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        const uint32_t x = s[w];
        s[w] = x - borrow;
        borrow = (x < borrow) ? 1u : 0u;
    }
    x2 = fe_one();
    z2 = fe_zero();
    x3 = q;
    z3 = fe_one();
    uint32_t swap = 0;
#pragma unroll 1
    for (int t = 251; t >= 0; --t) {
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

__global__ void __launch_bounds__(128) ladder_kernel(uint32_t* state, uint64_t* ns, const uint32_t* __restrict__ scalars,
                                                     uint32_t lanes, fe q) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= lanes) return;
    fe x2, z2, x3, z3;
    ladder_pair(scalars, lane, q, x2, z2, x3, z3);
    store_fe(state, 0, lane, lanes, x2);
    store_fe(state, 1, lane, lanes, z2);
    store_fe(state, 2, lane, lanes, x3);
    store_fe(state, 3, lane, lanes, z3);
    ns[lane] = 0;
}

// first_public_keys (mod.rs:212-228) on the GPU: u(k-8) and u(k) as 16
// canonical little-endian words per lane, the input of Backend::init.  One
// inversion of Z2 * Z3 serves both coordinates.
__global__ void __launch_bounds__(128) first_keys_kernel(uint32_t* __restrict__ upc, const uint32_t* __restrict__ scalars,
                                                         uint32_t lanes, fe q) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= lanes) return;
    fe x2, z2, x3, z3;
    ladder_pair(scalars, lane, q, x2, z2, x3, z3);
    const fe inv = fe_invert(fe_mul(z2, z3));
    const fe u_prev = fe_canon(fe_mul(x2, fe_mul(inv, z3)));
    const fe u_cur = fe_canon(fe_mul(x3, fe_mul(inv, z2)));
#pragma unroll
    for (int w = 0; w < 8; w++) {
        upc[(size_t)lane * 16 + w] = u_prev.v[w];
        upc[(size_t)lane * 16 + 8 + w] = u_cur.v[w];
    }
}

// ---- Primitive kernels for the field / hash microbench.

__device__ __forceinline__ fe load_words_drop255(const uint32_t* p) {
    fe r;
    const uint4* p4 = reinterpret_cast<const uint4*>(p);
    const uint4 lo = p4[0], hi = p4[1];
    r.v[0] = lo.x; r.v[1] = lo.y; r.v[2] = lo.z; r.v[3] = lo.w;
    r.v[4] = hi.x; r.v[5] = hi.y; r.v[6] = hi.z; r.v[7] = hi.w & 0x7fffffffu;
    return r;
}

// All 256 bits: an intermediate value of the 8-word representation.
__device__ __forceinline__ fe load_words(const uint32_t* p) {
    fe r;
    const uint4* p4 = reinterpret_cast<const uint4*>(p);
    const uint4 lo = p4[0], hi = p4[1];
    r.v[0] = lo.x; r.v[1] = lo.y; r.v[2] = lo.z; r.v[3] = lo.w;
    r.v[4] = hi.x; r.v[5] = hi.y; r.v[6] = hi.z; r.v[7] = hi.w;
    return r;
}

__device__ __forceinline__ void store_words(uint32_t* p, const fe& x) {
    uint4* p4 = reinterpret_cast<uint4*>(p);
    p4[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
    p4[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

__global__ void fe_op_kernel(int op, const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                             uint32_t* __restrict__ out, uint64_t count) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
        const fe x = load_words_drop255(a + 8 * i);
        fe r;
        if (op == 0) r = fe_mul(x, load_words_drop255(b + 8 * i));
        else if (op == 1) r = fe_sqr(x);
        else r = fe_invert(x);
        store_words(out + 8 * i, fe_canon(r));
    }
}

// Montgomery's trick over each group of `group` (<= 256) consecutive elements,
// one group per thread; the structure of the walk's batch inversion.
__global__ void fe_batch_invert_kernel(const uint32_t* __restrict__ a, uint32_t* __restrict__ out, uint64_t count,
                                       uint32_t group) {
    const uint64_t groups = (count + group - 1) / group;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < groups; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = g * group;
        const uint32_t len = (uint32_t)((count - base) < group ? (count - base) : group);
        // Prefix products go to the output buffer, then are overwritten.
        fe acc = fe_one();
        for (uint32_t i = 0; i < len; i++) {
            store_words(out + 8 * (base + i), acc);
            acc = fe_mul(acc, load_words_drop255(a + 8 * (base + i)));
        }
        fe inv = fe_invert(acc);
        for (int i = (int)len - 1; i >= 0; i--) {
            const fe pre = load_words(out + 8 * (base + i));
            store_words(out + 8 * (base + i), fe_canon(fe_mul(inv, pre)));
            inv = fe_mul(inv, load_words_drop255(a + 8 * (base + i)));
        }
    }
}

// Destination hashes of whole 64-byte public keys (both halves per element).
__global__ void address_chain_kernel(const uint32_t* __restrict__ pk, lxsha::AddrConsts ac, uint32_t* __restrict__ out,
                                     uint64_t count) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t u[8], hi[8], d[4];
#pragma unroll
        for (int w = 0; w < 8; w++) {
            u[w] = pk[16 * i + w];
            hi[w] = __byte_perm(pk[16 * i + 8 + w], 0, 0x0123);
        }
        lxsha::dest_hash(u, hi, ac, d);
        // Back to bytes in hash order: big-endian words.
#pragma unroll
        for (int w = 0; w < 4; w++) out[4 * i + w] = __byte_perm(d[w], 0, 0x0123);
    }
}

// ---- Integer-pipe throughput probes (the roofline's denominator).
// Each thread runs 8 independent dependency chains of one instruction class
// so that issue, not latency, is the limit; `sink` keeps the work alive.

// Operations counted per step and chain: kinds 2 and 5 issue two.
//   0 mad.lo.u32   1 mad.hi.u32   2 xor + shf   3 mad.wide.u32 (64-bit addend)
//   4 add.u32      5 mad.lo + xor (two pipes)   6 shf only   7 xor only
__global__ void __launch_bounds__(256) probe_kernel(int kind, uint32_t iters, uint32_t seed, uint32_t* sink) {
    uint32_t x[8], y[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        x[j] = seed + threadIdx.x * 8 + j;
        y[j] = x[j] ^ 0x55555555u;
    }
    const uint32_t m = seed | 1u, c = seed ^ 0x9e3779b9u;
#define LXK_PROBE(BODY)                                   \
    _Pragma("unroll 1") for (uint32_t i = 0; i < iters; i++) { \
        _Pragma("unroll") for (int r = 0; r < 16; r++) {   \
            _Pragma("unroll") for (int j = 0; j < 8; j++) { BODY; } \
        }                                                  \
    }
    switch (kind) {
        case 0: LXK_PROBE(asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[j]) : "r"(m), "r"(c))) break;
        case 1: LXK_PROBE(asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(x[j]) : "r"(m), "r"(c))) break;
        case 2:
            LXK_PROBE(asm volatile("xor.b32 %0, %0, %1;" : "+r"(x[j]) : "r"(c));
                      asm volatile("shf.r.wrap.b32 %0, %0, %0, 7;" : "+r"(x[j])))
            break;
        case 3:
            LXK_PROBE(asm volatile("{.reg .u64 t; mov.b64 t, {%0, %1}; mad.wide.u32 t, %0, %2, t; mov.b64 {%0, %1}, t;}"
                                   : "+r"(x[j]), "+r"(y[j]) : "r"(m)))
            break;
        // The neighbour operand keeps ptxas from folding repeated ops on one constant.
        case 4: LXK_PROBE(asm volatile("add.u32 %0, %0, %1;" : "+r"(x[j]) : "r"(x[(j + 1) & 7]))) break;
        case 5:
            LXK_PROBE(asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[j]) : "r"(m), "r"(c));
                      asm volatile("xor.b32 %0, %0, %1;" : "+r"(y[j]) : "r"(y[(j + 1) & 7])))
            break;
        case 6: LXK_PROBE(asm volatile("shf.r.wrap.b32 %0, %0, %0, 7;" : "+r"(x[j]))) break;
        default: LXK_PROBE(asm volatile("xor.b32 %0, %0, %1;" : "+r"(x[j]) : "r"(x[(j + 1) & 7]))) break;
    }
#undef LXK_PROBE
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) acc ^= x[j] ^ y[j];
    if (acc == 0x12345678u) sink[0] = acc;
}

}  // namespace lxk
