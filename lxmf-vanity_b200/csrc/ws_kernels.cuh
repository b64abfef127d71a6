// The grouped walk with its two halves on different warps (sm_100a).
//
// The grouped walk (group_kernels.cuh) alternates two phases per group: the
// field arithmetic, bound by the multiply-add pipe, and the SHA-256 chain of
// each key, bound by the integer ALU pipe.  With every warp of a block in the
// same phase, one pipe idles while the other is busy.  Here a block's warps
// are split by role and run both phases at once:
//
//   - F walker warps ("producers") each walk 32 lanes of the grouped walk.
//     In the backward pass of a group, iteration i yields the canonical u of
//     keys c + i and c - i for each lane; the warp writes them into the next
//     slot of its ring in shared memory (S slots) and arrives on the slot's
//     `full` barrier.  Its backward pass also carries the next group's
//     forward product (ws_produce), so only the inversion pauses the hand-over;
//   - C hash warps per walker warp ("consumers") each take every C-th slot of
//     that ring: wait on `full`, copy the two u's to registers, arrive on the
//     slot's `empty` barrier, then hash, compare and record hits exactly as
//     the plain kernel's emit_key does.
//
// The handshake uses shared-memory mbarriers (32 arrivals each: every thread
// of the arriving warp, so each thread's own stores are released by its own
// arrive).  Every wait is bounded: a wait that polls kWsWaitLimit times (with
// a 64 ns back-off, about a second) gives up, sets the launch's error flag
// and the block's abort flag, and every other waiting thread of the block
// then leaves too, so a launch always ends.  The host reports the flag as an
// error of the launch.
//
// Keys, hashes, hits and dumps are those of the grouped walk, key for key.
#pragma once
#include <cstdint>

#include "group_kernels.cuh"

namespace lxk {

constexpr uint32_t kWsWaitLimit = 1u << 24;

template <int F, int S>
struct WsShared {
    uint32_t u[F * S][2][8][32];  // [slot][side][word][lane]: side 0 key c + i, side 1 key c - i
    uint64_t n[F * S][2][32];     // walk index of each key
    uint32_t side0[F * S];        // 1 when side 0 holds a key (0 < i < M)
    unsigned long long full[F * S];
    unsigned long long empty[F * S];
    uint32_t abort;               // set by a wait that gave up: every waiter leaves
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

// Arrive (release, CTA scope: this thread's earlier shared-memory stores are
// visible to a thread whose wait on this phase succeeds).
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
    asm volatile(
        "{\n\t"
        ".reg .b64 st;\n\t"
        "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t"
        "}" ::"r"(smem_u32(b))
        : "memory");
}

// Whether the phase of parity `parity` has completed (acquire, CTA scope).
__device__ __forceinline__ bool mbar_test(unsigned long long* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of parity `parity`: false when this wait gave up
// or another thread of the block already did (the launch is then failed).
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, uint32_t parity, volatile uint32_t* abort,
                                          uint32_t* err) {
    for (uint32_t k = 0;; k++) {
        if (mbar_test(b, parity)) return true;
        if (*abort) return false;
        if (k >= kWsWaitLimit) {
            *abort = 1u;
            atomicOr(err, 1u);
            return false;
        }
        __nanosleep(64);
    }
}

template <int F, int S>
__device__ __forceinline__ void ws_put(WsShared<F, S>& sh, int k, int side, int lid, const fe& u, uint64_t n) {
#pragma unroll
    for (int w = 0; w < 8; w++) sh.u[k][side][w][lid] = u.v[w];
    sh.n[k][side][lid] = n;
}

// Hands the canonical u of keys c + i (when side0) and c - i to the ring:
// slot of backward iteration j (counted over the whole launch) p * S + j % S,
// in round j / S.  False when a wait gave up.
template <int F, int S>
__device__ __forceinline__ bool ws_hand(WsShared<F, S>& sh, int p, int lid, uint32_t j, bool side0, const fe& up,
                                        const fe& um, uint64_t c, int i, uint32_t* err) {
    const fe u0 = fe_canon(up), u1 = fe_canon(um);
    const int k = p * S + (int)(j % S);
    const uint32_t round = j / S;
    if (round > 0 && !mbar_wait(&sh.empty[k], (round - 1) & 1u, &sh.abort, err)) return false;
    if (side0) ws_put(sh, k, 0, lid, u0, c + (uint64_t)i);
    ws_put(sh, k, 1, lid, u1, c - (uint64_t)i);
    if (lid == 0) sh.side0[k] = side0 ? 1u : 0u;
    mbar_arrive(&sh.full[k]);
    return true;
}

// One walker warp's lanes: `groups` groups from centre (uc, vc) at walk index
// n.  The order of the Montgomery product is e_1 .. e_M, then e_0 (the
// denominator of the step to the next centre C + J), so the backward pass
// yields 1/e_0 first: the next centre is known at the start of the pass, and
// each backward iteration also does one step of the next group's forward
// product.  The walker warp then hands keys to the hash warps through the
// whole group except its one inversion, instead of pausing for the forward
// pass (about a fifth of its work).  pre[g][k] = d_1 ... d_(k-1) of buffer g.
template <int M, int F, int S, class Table>
__device__ __forceinline__ bool ws_produce(fe& uc, fe& vc, uint64_t& n, uint32_t groups, const Table& t,
                                           WsShared<F, S>& sh, int p, int lid, uint32_t* err) {
    fe pre[2][M + 2];
    fe cA = fe_zero();
    cA.v[0] = LXK_A;
    // The first group's forward product, in full.
    fe acc = fe_one();
#pragma unroll 1
    for (int k = 1; k <= M; ++k) {
        pre[0][k] = acc;
        acc = fe_mul(acc, fe_sub(t.u[k], uc));
    }
    pre[0][M + 1] = acc;
    acc = fe_mul(acc, fe_sub(t.u[0], uc));
    int cur = 0;
    uint32_t j = 0;
#pragma unroll 1
    for (uint32_t it = 0; it < groups; ++it) {
        const bool more = it + 1 < groups;  // uniform: the next group's forward product rides along
        fe inv = fe_invert(acc);
        const uint64_t c = n + M;
        const fe s0 = fe_add(uc, cA);
        // The step to the next centre, C' = C + J (table entry 0), first.
        fe un, vn;
        {
            const fe tu = t.u[0], tv = t.v[0];
            const fe inv0 = fe_mul(inv, pre[cur][M + 1]);
            inv = fe_mul(inv, fe_sub(tu, uc));
            const fe lp = fe_mul(fe_sub(tv, vc), inv0);
            un = fe_sub(fe_sqr(lp), fe_add(s0, tu));
            vn = fe_sub(fe_mul(lp, fe_sub(uc, un)), vc);
        }
        fe accn = fe_one();
#pragma unroll 1
        for (int i = M; i >= 1; --i, ++j) {
            const fe tu = t.u[i], tv = t.v[i];
            const fe invi = fe_mul(inv, pre[cur][i]);
            inv = fe_mul(inv, fe_sub(tu, uc));
            const fe s = fe_add(s0, tu);
            const fe up = fe_sub(fe_sqr(fe_mul(fe_sub(tv, vc), invi)), s);  // C + T_i
            const fe um = fe_sub(fe_sqr(fe_mul(fe_add(tv, vc), invi)), s);  // C - T_i
            if (more) {
                const int k = M + 1 - i;  // 1 .. M
                pre[cur ^ 1][k] = accn;
                accn = fe_mul(accn, fe_sub(t.u[k], un));
            }
            if (!ws_hand(sh, p, lid, j, i < M, up, um, c, i, err)) return false;
        }
        // The centre itself, key c.
        if (!ws_hand(sh, p, lid, j, false, uc, uc, c, 0, err)) return false;
        ++j;
        if (more) {
            pre[cur ^ 1][M + 1] = accn;
            acc = fe_mul(accn, fe_sub(t.u[0], un));
        }
        uc = un;
        vc = vn;
        n += 2 * M;
        cur ^= 1;
    }
    return true;
}

// One hash warp: iterations j = c, c + C, ... of walker warp p's ring.
template <int F, int C, int S, bool DUMP>
__device__ __forceinline__ void ws_consume(WsShared<F, S>& sh, int p, int c, int lid, const EmitArgs& em,
                                           uint32_t lane, bool active, uint64_t key0, uint32_t total, uint32_t* err) {
    volatile uint32_t* abort = &sh.abort;
#pragma unroll 1
    for (uint32_t j = (uint32_t)c; j < total; j += C) {
        const int k = p * S + (int)(j % S);
        if (!mbar_wait(&sh.full[k], (j / S) & 1u, abort, err)) return;
        fe u0, u1;
#pragma unroll
        for (int w = 0; w < 8; w++) {
            u0.v[w] = sh.u[k][0][w][lid];
            u1.v[w] = sh.u[k][1][w][lid];
        }
        const uint64_t n0 = sh.n[k][0][lid], n1 = sh.n[k][1][lid];
        const bool side0 = sh.side0[k] != 0;
        mbar_arrive(&sh.empty[k]);
        if (active) {
            if (side0) emit_key<DUMP>(em, lane, n0, key0, u0);
            emit_key<DUMP>(em, lane, n1, key0, u1);
        }
    }
}

// Launch parameters: the grouped walk's, plus the launch's error flag.
template <int M>
struct WsArgs {
    GroupArgsFor<M> g;
    uint32_t* err;  // set to 1 when a wait gave up
};

// F walker warps and F * C hash warps per block; F * 32 lanes per block.
// Threads of walker lanes past the last lane walk a copy of the last lane and
// neither emit nor store.  PREGS / QREGS (0: no change): registers per thread
// the walker and hash warps move to with setmaxnreg after the split.  The
// split must add up to no more than the block's launch registers (threads x
// the kernel's register count), else the walkers' increase would wait for
// registers that never come; the host checks that sum before the first launch
// (ws_regsplit_fits).  The walker warps must fill whole warpgroups.
template <int M, int F, int C, int S, bool DUMP, int PREGS = 0, int QREGS = 0>
static __global__ void __launch_bounds__(32 * F * (1 + C), 1) group_walk_ws_kernel(const __grid_constant__ WsArgs<M> a) {
    extern __shared__ __align__(16) unsigned char ws_smem[];
    WsShared<F, S>& sh = *reinterpret_cast<WsShared<F, S>*>(ws_smem);
    if (threadIdx.x == 0) {
        for (int k = 0; k < F * S; k++) {
            mbar_init(&sh.full[k], 32);
            mbar_init(&sh.empty[k], 32);
        }
        sh.abort = 0;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lid = threadIdx.x & 31;
    const int p = warp < F ? warp : (warp - F) / C;
    const uint32_t tid = blockIdx.x * (32 * F) + 32 * p + lid;
    const bool active = tid < a.g.lanes;
    const uint32_t lane = active ? tid : a.g.lanes - 1;
    if (warp < F) {
        if constexpr (PREGS > 0) asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(PREGS));
        fe uc = load_fe(a.g.state, 0, lane, a.g.lanes);
        fe vc = load_fe(a.g.state, 1, lane, a.g.lanes);
        uint64_t n = a.g.ns[lane];
        const bool ok = ws_produce<M, F, S>(uc, vc, n, a.g.iters, table_of(a.g), sh, p, lid, a.err);
        if (ok && active) {
            store_fe(a.g.state, 0, lane, a.g.lanes, uc);
            store_fe(a.g.state, 1, lane, a.g.lanes, vc);
            a.g.ns[lane] = n;
        }
    } else {
        if constexpr (QREGS > 0) asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(QREGS));
        // Read before this warp's first arrive: the walker warp's final store
        // of ns comes after it has seen that arrive.
        const uint64_t key0 = a.g.ns[lane];
        ws_consume<F, C, S, DUMP>(sh, p, (warp - F) % C, lid, a.g.em, lane, active, key0,
                                  a.g.iters * (uint32_t)(M + 1), a.err);
    }
}

}  // namespace lxk
