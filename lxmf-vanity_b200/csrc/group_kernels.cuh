// The grouped affine walk (sm_100a): the same keys as the x-only walk, with
// about half the field work per key.
//
// Curve25519 in Montgomery form, v^2 = u^3 + A u^2 + u, A = 486662.  Every
// point here is a multiple of Q = 8B, with v(Q) fixed to the even square
// root, so a lane's key with walk index n is the point (k/8 + n) Q and its
// public key is that point's u.  A group is G = 2M keys: walk indices
// c-M .. c+M-1 around a centre C = (k/8 + c) Q kept affine (u_C, v_C):
//
//   key c +- i  =  C +- T_i,  T_i = i Q from a table (i = 1..M),
//   affine addition:  l = (v_T -+ v_C) / (u_T - u_C),  u = l^2 - A - u_C - u_T.
//
// C + T_i and C - T_i share the denominator u_T - u_C, so one batch inversion
// (Montgomery's trick) over the M denominators and the step to the next
// centre, C' = C + J with J = 2M Q, serves all 2M keys.  Per group:
// (5M + 15) M + (2M + 254) S, i.e. about 2.6 M + 2.5 S per key at G = 128,
// against 8 M + 4 S for the x-only walk (G = B = 128).  The lane's local
// buffer holds only the M prefix products (the denominators are recomputed
// from the table on the way back).
//
// Lane state in HBM: u_C, v_C (2 x 32 bytes, word-major) and the walk index
// of the group's first key.
#pragma once
#include <cstdint>
#include <type_traits>

#include "walk_kernels.cuh"

namespace lxk {

// 2A, for the y-coordinate recovery.
#define LXK_TWO_A 973324u
#define LXK_A 486662u

template <int M>
struct GroupTable {
    fe u[M + 1];  // [0]: J = 2M Q; [i]: i Q
    fe v[M + 1];
};

template <int M>
struct GroupArgs {
    uint32_t* state;  // [16][lanes]: u_C, v_C
    uint64_t* ns;     // [lanes]: walk index of the first key of the lane's next group (centre - M)
    uint32_t lanes;
    uint32_t iters;   // groups per lane in this launch
    EmitArgs em;
    GroupTable<M> t;
};

// G = 1024 (M = 512): the table (2 x 513 points, 33 KB) no longer fits the
// kernel parameter block (32 KB), so it lives in constant memory, where the
// warps read it through the same constant cache.  It depends on nothing but
// M, so every handle on a device shares it; lxmfv_open writes it there.
constexpr int kConstTableM = 512;
static __device__ __constant__ fe c_group_u[kConstTableM + 1];
static __device__ __constant__ fe c_group_v[kConstTableM + 1];
struct ConstTableU {
    __device__ __forceinline__ fe operator[](int i) const { return c_group_u[i]; }
};
struct ConstTableV {
    __device__ __forceinline__ fe operator[](int i) const { return c_group_v[i]; }
};
struct ConstGroupTable {
    ConstTableU u;
    ConstTableV v;
};
struct GroupArgsConst {
    uint32_t* state;
    uint64_t* ns;
    uint32_t lanes;
    uint32_t iters;
    EmitArgs em;
};
template <int M>
__device__ __forceinline__ const GroupTable<M>& table_of(const GroupArgs<M>& a) { return a.t; }
__device__ __forceinline__ ConstGroupTable table_of(const GroupArgsConst&) { return ConstGroupTable{}; }
// The launch parameters of the grouped walk at M: the table travels in them
// up to M = 256, and sits in constant memory above.
template <int M>
using GroupArgsFor = typename std::conditional<(M > 256), GroupArgsConst, GroupArgs<M>>::type;

// y-coordinate recovery on a Montgomery curve (Okeya and Sakurai, CHES 2001;
// the form of Costello and Smith, "Montgomery curves and their arithmetic",
// Algorithm 5): from P = (xp, yp) affine, (X1:Z1) = sP and (X2:Z2) = (s+1)P,
// the projective (X:Y:Z) of sP.
__device__ __forceinline__ void recover_y(const fe& xp, const fe& yp, const fe& X1, const fe& Z1, const fe& X2,
                                          const fe& Z2, fe& X, fe& Y, fe& Z) {
    fe v1 = fe_mul(xp, Z1);
    fe v2 = fe_add(X1, v1);
    fe v3 = fe_sub(X1, v1);
    v3 = fe_mul(fe_sqr(v3), X2);
    v1 = fe_mul_small(Z1, LXK_TWO_A);
    v2 = fe_add(v2, v1);
    const fe v4 = fe_add(fe_mul(xp, X1), Z1);
    v2 = fe_mul(v2, v4);
    v1 = fe_mul(v1, Z1);
    v2 = fe_mul(fe_sub(v2, v1), Z2);
    Y = fe_sub(v2, v3);
    v1 = fe_mul(fe_mul(fe_add(yp, yp), Z1), Z2);
    X = fe_mul(v1, X1);
    Z = fe_mul(v1, Z1);
}

__device__ __forceinline__ void to_affine(const fe& X, const fe& Y, const fe& Z, fe& u, fe& v) {
    const fe zi = fe_invert(Z);
    u = fe_canon(fe_mul(X, zi));
    v = fe_canon(fe_mul(Y, zi));
}

// The table: thread i computes i Q (i = 1..M) and thread 0 computes J = 2M Q,
// affine and canonical, into tu / tv ([M + 1] each).
static __global__ void group_table_kernel(fe* tu, fe* tv, uint32_t m, fe q, fe vq) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    uint32_t s[8] = {i == 0 ? 2 * m : i, 0, 0, 0, 0, 0, 0, 0};
    fe x2, z2, x3, z3, X, Y, Z;
    ladder(s, 32, q, x2, z2, x3, z3);
    recover_y(q, vq, x2, z2, x3, z3, X, Y, Z);
    to_affine(X, Y, Z, tu[i], tv[i]);
}

// Start from scalars: C = (k/8 + M) Q, the centre of the first group (walk
// indices 0 .. 2M-1).
static __global__ void __launch_bounds__(128) group_start_kernel(uint32_t* state, uint64_t* ns,
                                                          const uint32_t* __restrict__ scalars, uint32_t lanes,
                                                          uint32_t m, fe q, fe vq) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= lanes) return;
    uint32_t s[8];
    scalar_over_8(scalars, lane, (int)m, s);
    fe x2, z2, x3, z3, X, Y, Z, u, v;
    ladder(s, 253, q, x2, z2, x3, z3);
    recover_y(q, vq, x2, z2, x3, z3, X, Y, Z);
    to_affine(X, Y, Z, u, v);
    store_fe(state, 0, lane, lanes, u);
    store_fe(state, 1, lane, lanes, v);
    ns[lane] = 0;
}

// Start from Backend::init's u(k-8), u(k): y of P = kB = (k/8) Q is recovered
// with -Q (P - Q is known, not P + Q), then C = P + T_M (tm = M Q).
static __global__ void __launch_bounds__(128) group_init_kernel(uint32_t* state, uint64_t* ns,
                                                         const uint32_t* __restrict__ upc, uint32_t lanes, fe q,
                                                         fe vq_neg, fe tmu, fe tmv) {
    const uint32_t lane = blockIdx.x * blockDim.x + threadIdx.x;
    if (lane >= lanes) return;
    fe um8, uk;
#pragma unroll
    for (int w = 0; w < 8; w++) {
        um8.v[w] = upc[(size_t)lane * 16 + w];
        uk.v[w] = upc[(size_t)lane * 16 + 8 + w];
    }
    um8.v[7] &= 0x7fffffffu;
    uk.v[7] &= 0x7fffffffu;
    fe X, Y, Z, pu, pv;
    recover_y(q, vq_neg, uk, fe_one(), um8, fe_one(), X, Y, Z);
    to_affine(X, Y, Z, pu, pv);
    fe cA = fe_zero();
    cA.v[0] = LXK_A;
    const fe l = fe_mul(fe_sub(tmv, pv), fe_invert(fe_sub(tmu, pu)));
    const fe u = fe_canon(fe_sub(fe_sqr(l), fe_add(fe_add(pu, tmu), cA)));
    const fe v = fe_canon(fe_sub(fe_mul(l, fe_sub(pu, u)), pv));
    store_fe(state, 0, lane, lanes, u);
    store_fe(state, 1, lane, lanes, v);
    ns[lane] = 0;
}

// `groups` groups of one lane's walk from centre (uc, vc) at walk index n
// (the first key of the next group); emit(u, key) receives every key's
// canonical u.  Shared by the plain walk and the pool's persistent kernel.
// SYNC: a block barrier after each group keeps the block's warps in the same
// phase of the walk, so that they share the instruction cache's working set
// (one phase's code instead of all of it); every thread of the block must
// then call this with the same `groups`.
template <int M, bool SYNC, class Table, class Emit>
__device__ __forceinline__ void walk_groups(fe& uc, fe& vc, uint64_t& n, uint32_t groups, const Table& t,
                                            const Emit& emit) {
    fe pre[M + 1];
    fe cA = fe_zero();
    cA.v[0] = LXK_A;
#pragma unroll 1
    for (uint32_t it = 0; it < groups; ++it) {
        // Denominators e_0 = u_J - u_C, e_i = u_{T_i} - u_C; pre[i] = e_0 ... e_{i-1}.
        fe acc = fe_sub(t.u[0], uc);
#pragma unroll 1
        for (int i = 1; i <= M; ++i) {
            pre[i] = acc;
            acc = fe_mul(acc, fe_sub(t.u[i], uc));
        }
        fe inv = fe_invert(acc);
        const uint64_t c = n + M;
        const fe s0 = fe_add(uc, cA);
        fe vnext = vc;
#pragma unroll 1
        for (int i = M; i >= 0; --i) {
            const fe tu = t.u[i], tv = t.v[i];
            fe invi = inv;  // 1 / e_i
            if (i > 0) {
                invi = fe_mul(inv, pre[i]);
                inv = fe_mul(inv, fe_sub(tu, uc));
            }
            const fe s = fe_add(s0, tu);
            const fe lp = fe_mul(fe_sub(tv, vc), invi);
            const fe up = fe_sub(fe_sqr(lp), s);  // C + T_i (for i = 0: the next centre C + J)
            fe um;
            if (i > 0) {
                const fe lm = fe_mul(fe_add(tv, vc), invi);
                um = fe_sub(fe_sqr(lm), s);       // C - T_i
            } else {
                um = uc;                          // C itself
                vnext = fe_sub(fe_mul(lp, fe_sub(uc, up)), vc);
            }
#pragma unroll 1
            for (int side = 0; side < 2; ++side) {
                // side 0: key c + i (only 0 < i < M: c + M is the next group's);
                // side 1: key c - i (i = 0: the centre).
                if (side == 1 || (i > 0 && i < M)) {
                    const fe u = fe_canon(side ? um : up);
                    emit(u, side ? c - (uint64_t)i : c + (uint64_t)i);
                }
            }
            if (i == 0) {
                uc = up;
                vc = vnext;
            }
        }
        n += 2 * M;
        if (SYNC) __syncthreads();
    }
}

// The plain search's emission: one prefix for every lane of the launch.
template <bool DUMP>
struct LaneEmit {
    const EmitArgs& em;
    uint32_t lane;
    uint64_t key0;
    bool active;
    __device__ __forceinline__ void operator()(const fe& u, uint64_t key) const {
        if (active) emit_key<DUMP>(em, lane, key, key0, u);
    }
};

// Threads past the last lane walk a copy of the last lane and neither emit
// nor store (with SYNC they must still reach every barrier).
template <int M, int BLOCK, int MINB, bool SYNC, bool DUMP, class Args = GroupArgsFor<M>>
static __global__ void __launch_bounds__(BLOCK, MINB) group_walk_kernel(const __grid_constant__ Args a) {
    const uint32_t tid = blockIdx.x * BLOCK + threadIdx.x;
    if (!SYNC && tid >= a.lanes) return;
    const bool active = tid < a.lanes;
    const uint32_t lane = active ? tid : a.lanes - 1;
    fe uc = load_fe(a.state, 0, lane, a.lanes);
    fe vc = load_fe(a.state, 1, lane, a.lanes);
    const uint64_t key0 = a.ns[lane];
    uint64_t n = key0;
    const LaneEmit<DUMP> emit{a.em, lane, key0, active};
    walk_groups<M, SYNC>(uc, vc, n, a.iters, table_of(a), emit);
    if (active) {
        store_fe(a.state, 0, lane, a.lanes, uc);
        store_fe(a.state, 1, lane, a.lanes, vc);
        a.ns[lane] = n;
    }
}

}  // namespace lxk
