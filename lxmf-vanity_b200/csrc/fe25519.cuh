// GF(2^255 - 19) on 8 x 32-bit limbs for sm_100a.
//
// Replaces the reference's 10-limb signed radix-2^25.5 field (src/gpu/
// common.h:25-174).  Representation: an element is any 256-bit value x
// (8 little-endian 32-bit words) standing for x mod p.  2^256 = 38 (mod p),
// so sums and products fold their overflow back with a multiply by 38; only
// fe_canon maps to the canonical [0, p) encoding (the reference's
// fe_to_words, common.h:145-174).  Multiplies are 32x32->64 IMAD chains with
// explicit carries (fe25519_ptx.cuh, generated by gen_fe_ptx.py).
#pragma once
#include <cstdint>

struct __align__(16) fe {
    uint32_t v[8];
};

#include "fe25519_ptx.cuh"

// The multiply and the square are out of line: one body each in the binary,
// reached by a call.  Measured on B200 against the bodies inlined at every
// call site: the grouped walk +1.5% and the pool kernel +2% (smaller loops for
// the instruction caches), the x-only walk -2.3% (four times the multiplies
// per key, so the calls cost more than the code size saves).
static __device__ __noinline__ fe fe_mul(const fe& a, const fe& b) {
    fe o;
    fe_mul_ptx(o, a, b);
    return o;
}

static __device__ __noinline__ fe fe_sqr(const fe& a) {
    fe o;
    fe_sqr_ptx(o, a);
    return o;
}

__device__ __forceinline__ fe fe_zero() {
    fe o;
#pragma unroll
    for (int i = 0; i < 8; i++) o.v[i] = 0;
    return o;
}

__device__ __forceinline__ fe fe_one() {
    fe o = fe_zero();
    o.v[0] = 1;
    return o;
}

// a + b; a carry out of 2^256 is worth 38, and a second carry can only leave
// a value below 76, so the last fold needs no chain.  Adding 38 to limb 0
// carries into limb 1 with probability below 2^-26 on uniform inputs, so that
// chain is a branch: the common case skips seven carry steps.
__device__ __forceinline__ fe fe_add(const fe& a, const fe& b) {
    fe o;
    asm("{\n\t"
        ".reg .u32 c, t;\n\t"
        ".reg .pred p;\n\t"
        "add.cc.u32 %0, %8, %16;\n\t"
        "addc.cc.u32 %1, %9, %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.cc.u32 %7, %15, %23;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "mul.lo.u32 t, c, 38;\n\t"
        "add.cc.u32 %0, %0, t;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "setp.eq.u32 p, c, 0;\n\t"
        "@p bra ADDED;\n\t"
        "add.cc.u32 %1, %1, 1;\n\t"
        "addc.cc.u32 %2, %2, 0;\n\t"
        "addc.cc.u32 %3, %3, 0;\n\t"
        "addc.cc.u32 %4, %4, 0;\n\t"
        "addc.cc.u32 %5, %5, 0;\n\t"
        "addc.cc.u32 %6, %6, 0;\n\t"
        "addc.cc.u32 %7, %7, 0;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "mad.lo.u32 %0, c, 38, %0;\n\t"
        "ADDED:\n\t"
        "}"
        : "=r"(o.v[0]), "=r"(o.v[1]), "=r"(o.v[2]), "=r"(o.v[3]), "=r"(o.v[4]), "=r"(o.v[5]), "=r"(o.v[6]),
          "=r"(o.v[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    return o;
}

// a - b; a borrow past 0 added 2^256 = 38, so 38 is taken off again (twice
// at most: after a second borrow the value is at least 2^256 - 38).  As in
// fe_add, the borrow out of limb 0 is rare and its chain is a branch.
__device__ __forceinline__ fe fe_sub(const fe& a, const fe& b) {
    fe o;
    asm("{\n\t"
        ".reg .u32 c, t;\n\t"
        ".reg .pred p;\n\t"
        "sub.cc.u32 %0, %8, %16;\n\t"
        "subc.cc.u32 %1, %9, %17;\n\t"
        "subc.cc.u32 %2, %10, %18;\n\t"
        "subc.cc.u32 %3, %11, %19;\n\t"
        "subc.cc.u32 %4, %12, %20;\n\t"
        "subc.cc.u32 %5, %13, %21;\n\t"
        "subc.cc.u32 %6, %14, %22;\n\t"
        "subc.cc.u32 %7, %15, %23;\n\t"
        "subc.u32 c, 0, 0;\n\t"
        "and.b32 t, c, 38;\n\t"
        "sub.cc.u32 %0, %0, t;\n\t"
        "subc.u32 c, 0, 0;\n\t"
        "setp.eq.u32 p, c, 0;\n\t"
        "@p bra SUBBED;\n\t"
        "sub.cc.u32 %1, %1, 1;\n\t"
        "subc.cc.u32 %2, %2, 0;\n\t"
        "subc.cc.u32 %3, %3, 0;\n\t"
        "subc.cc.u32 %4, %4, 0;\n\t"
        "subc.cc.u32 %5, %5, 0;\n\t"
        "subc.cc.u32 %6, %6, 0;\n\t"
        "subc.cc.u32 %7, %7, 0;\n\t"
        "subc.u32 c, 0, 0;\n\t"
        "and.b32 t, c, 38;\n\t"
        "sub.u32 %0, %0, t;\n\t"
        "SUBBED:\n\t"
        "}"
        : "=r"(o.v[0]), "=r"(o.v[1]), "=r"(o.v[2]), "=r"(o.v[3]), "=r"(o.v[4]), "=r"(o.v[5]), "=r"(o.v[6]),
          "=r"(o.v[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    return o;
}

// a * k for a small constant k (k < 2^26), e.g. (A - 2) / 4 = 121665.
__device__ __forceinline__ fe fe_mul_small(const fe& a, uint32_t k) {
    fe o;
    asm("{\n\t"
        ".reg .u32 c, t;\n\t"
        "mul.lo.u32 %0, %8, %16;\n\t"
        "mul.lo.u32 %1, %9, %16;\n\t"
        "mul.lo.u32 %2, %10, %16;\n\t"
        "mul.lo.u32 %3, %11, %16;\n\t"
        "mul.lo.u32 %4, %12, %16;\n\t"
        "mul.lo.u32 %5, %13, %16;\n\t"
        "mul.lo.u32 %6, %14, %16;\n\t"
        "mul.lo.u32 %7, %15, %16;\n\t"
        "mad.hi.cc.u32 %1, %8, %16, %1;\n\t"
        "madc.hi.cc.u32 %2, %9, %16, %2;\n\t"
        "madc.hi.cc.u32 %3, %10, %16, %3;\n\t"
        "madc.hi.cc.u32 %4, %11, %16, %4;\n\t"
        "madc.hi.cc.u32 %5, %12, %16, %5;\n\t"
        "madc.hi.cc.u32 %6, %13, %16, %6;\n\t"
        "madc.hi.cc.u32 %7, %14, %16, %7;\n\t"
        "madc.hi.u32 c, %15, %16, 0;\n\t"
        "mul.lo.u32 t, c, 38;\n\t"
        "add.cc.u32 %0, %0, t;\n\t"
        "addc.cc.u32 %1, %1, 0;\n\t"
        "addc.cc.u32 %2, %2, 0;\n\t"
        "addc.cc.u32 %3, %3, 0;\n\t"
        "addc.cc.u32 %4, %4, 0;\n\t"
        "addc.cc.u32 %5, %5, 0;\n\t"
        "addc.cc.u32 %6, %6, 0;\n\t"
        "addc.cc.u32 %7, %7, 0;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "mad.lo.u32 %0, c, 38, %0;\n\t"
        "}"
        : "=r"(o.v[0]), "=r"(o.v[1]), "=r"(o.v[2]), "=r"(o.v[3]), "=r"(o.v[4]), "=r"(o.v[5]), "=r"(o.v[6]),
          "=r"(o.v[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(k));
    return o;
}

// The canonical representative in [0, p): fold bit 255 (2^255 = 19), which
// leaves x < 2^255 + 19 < 2p, then subtract p once when x + 19 reaches 2^255.
__device__ __forceinline__ fe fe_canon(const fe& a) {
    fe o;
    asm("{\n\t"
        ".reg .u32 t, x0, x1, x2, x3, x4, x5, x6, x7, y0, y1, y2, y3, y4, y5, y6, y7, m;\n\t"
        "shr.u32 t, %15, 31;\n\t"
        "and.b32 x7, %15, 0x7fffffff;\n\t"
        "mul.lo.u32 t, t, 19;\n\t"
        "add.cc.u32 x0, %8, t;\n\t"
        "addc.cc.u32 x1, %9, 0;\n\t"
        "addc.cc.u32 x2, %10, 0;\n\t"
        "addc.cc.u32 x3, %11, 0;\n\t"
        "addc.cc.u32 x4, %12, 0;\n\t"
        "addc.cc.u32 x5, %13, 0;\n\t"
        "addc.cc.u32 x6, %14, 0;\n\t"
        "addc.u32 x7, x7, 0;\n\t"
        "add.cc.u32 y0, x0, 19;\n\t"
        "addc.cc.u32 y1, x1, 0;\n\t"
        "addc.cc.u32 y2, x2, 0;\n\t"
        "addc.cc.u32 y3, x3, 0;\n\t"
        "addc.cc.u32 y4, x4, 0;\n\t"
        "addc.cc.u32 y5, x5, 0;\n\t"
        "addc.cc.u32 y6, x6, 0;\n\t"
        "addc.u32 y7, x7, 0;\n\t"
        "shr.s32 m, y7, 31;\n\t"
        "and.b32 y7, y7, 0x7fffffff;\n\t"
        "xor.b32 t, x0, y0;\n\t and.b32 t, t, m;\n\t xor.b32 %0, x0, t;\n\t"
        "xor.b32 t, x1, y1;\n\t and.b32 t, t, m;\n\t xor.b32 %1, x1, t;\n\t"
        "xor.b32 t, x2, y2;\n\t and.b32 t, t, m;\n\t xor.b32 %2, x2, t;\n\t"
        "xor.b32 t, x3, y3;\n\t and.b32 t, t, m;\n\t xor.b32 %3, x3, t;\n\t"
        "xor.b32 t, x4, y4;\n\t and.b32 t, t, m;\n\t xor.b32 %4, x4, t;\n\t"
        "xor.b32 t, x5, y5;\n\t and.b32 t, t, m;\n\t xor.b32 %5, x5, t;\n\t"
        "xor.b32 t, x6, y6;\n\t and.b32 t, t, m;\n\t xor.b32 %6, x6, t;\n\t"
        "xor.b32 t, x7, y7;\n\t and.b32 t, t, m;\n\t xor.b32 %7, x7, t;\n\t"
        "}"
        : "=r"(o.v[0]), "=r"(o.v[1]), "=r"(o.v[2]), "=r"(o.v[3]), "=r"(o.v[4]), "=r"(o.v[5]), "=r"(o.v[6]),
          "=r"(o.v[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]));
    return o;
}

// The ref10 addition chain for z^(p-2) (254 squarings, 11 multiplications;
// the chain of the reference's fe_invert, common.h:115-128), as a table that
// a loop walks, so that its code holds one square and one multiply instead of
// 265 inlined bodies.  After z2 = z^2, step s squares the running value
// kSq[s] times and multiplies it by operand kOp[s]; kSave[s] names the slot
// that keeps the result for a later step.
// Operands: 0 z, 1 z2, 2 z9, 3 z11, 4 z^(2^10-1), 5 z^(2^50-1), 6 the step's
// own input (z^(2^5-1), z^(2^10-1), ... doubling the run of ones).
__device__ __constant__ uint8_t kInvSq[11] = {2, 0, 1, 5, 10, 20, 10, 50, 100, 50, 5};
__device__ __constant__ uint8_t kInvOp[11] = {0, 1, 2, 6, 6, 6, 4, 6, 6, 5, 3};
__device__ __constant__ uint8_t kInvSave[11] = {2, 3, 0, 4, 0, 0, 5, 0, 0, 0, 0};

// z^(p-2).  0 maps to 0.  (static: each translation unit has its own copy.)
static __device__ __noinline__ fe fe_invert(fe z) {
    fe z2 = fe_sqr(z);
    fe z9 = z, z11 = z, z10 = z, z50 = z;
    fe t = z2;
#pragma unroll 1
    for (int s = 0; s < 11; s++) {
        const fe base = t;
        const int n = kInvSq[s];
#pragma unroll 1
        for (int i = 0; i < n; i++) t = fe_sqr(t);
        const int op = kInvOp[s];
        fe m = base;
        m = (op == 0) ? z : m;
        m = (op == 1) ? z2 : m;
        m = (op == 2) ? z9 : m;
        m = (op == 3) ? z11 : m;
        m = (op == 4) ? z10 : m;
        m = (op == 5) ? z50 : m;
        t = fe_mul(t, m);
        const int sv = kInvSave[s];
        z9 = (sv == 2) ? t : z9;
        z11 = (sv == 3) ? t : z11;
        z10 = (sv == 4) ? t : z10;
        z50 = (sv == 5) ? t : z50;
    }
    return t;
}

// Conditional swap by mask (m all ones or all zeros), without branches.
__device__ __forceinline__ void fe_cswap(fe& a, fe& b, uint32_t m) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint32_t t = m & (a.v[i] ^ b.v[i]);
        a.v[i] ^= t;
        b.v[i] ^= t;
    }
}
