// Primitive kernels: the field and hash microbench, and the integer-pipe
// throughput probes that give the roofline its denominators.
#pragma once
#include <cstdint>

#include "fe25519.cuh"
#include "sha256_lxmf.cuh"

namespace lxk {

// 8 words with bit 255 dropped, as the reference's fe_from_words reads them
// (common.h:131-142).
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

static __global__ void fe_op_kernel(int op, const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
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
static __global__ void fe_batch_invert_kernel(const uint32_t* __restrict__ a, uint32_t* __restrict__ out, uint64_t count,
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
static __global__ void address_chain_kernel(const uint32_t* __restrict__ pk, lxsha::AddrConsts ac, uint32_t* __restrict__ out,
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

// Each thread runs 8 independent dependency chains of one instruction class
// so that issue, not latency, is the limit; `sink` keeps the work alive.
// Operations counted per step and chain: kinds 2 and 5 issue two.
//   0 mad.lo.u32   1 mad.hi.u32   2 xor + shf   3 mad.wide.u32 (64-bit addend)
//   4 add.u32      5 mad.lo + xor (two pipes)   6 shf only   7 xor only
static __global__ void __launch_bounds__(256) probe_kernel(int kind, uint32_t iters, uint32_t seed, uint32_t* sink) {
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
