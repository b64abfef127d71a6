// liblxmfv: the C ABI of include/lxmfv.h over the sm_100a kernels.
//
// Replaces the reference's CUDA backend (src/gpu/cuda.rs): where that
// compiles common.h with NVRTC at start-up and, on every launch, copies four
// small arrays to the device and allocates three buffers (cuda.rs:93-101),
// this library is compiled ahead of time for sm_100a, passes the launch
// arguments by value in the kernel's parameter block, and keeps the hit
// queue and dump buffers allocated for the handle's lifetime.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "../../include/lxmfv.h"
#include "group_kernels.cuh"
#include "prim_kernels.cuh"
#include "walk_kernels.cuh"
#include "ws_kernels.cuh"

struct lxmfv_handle {
    int device = 0;
    int sms = 0;
    int cc_major = 0, cc_minor = 0;
    std::string name;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t walk = LXMFV_WALK_GROUP;
    uint32_t lanes = 0;
    uint32_t batch = 64;  // keys per inversion: B (x-only walk) or G = 2M (grouped walk)
    uint32_t block = 256;
    bool sync = false;    // grouped walk: block barrier after each group
    bool low_regs = false;  // LXMFV_FLAG_REGCAP_80
    bool ws = false;        // LXMFV_FLAG_WARP_SPEC: walker and hash warps
    uint32_t* d_err = nullptr;  // set by a warp-specialised launch whose wait gave up
    uint32_t* d_state = nullptr;
    uint64_t* d_ns = nullptr;
    uint32_t* d_hit_count = nullptr;
    lxk::Hit* d_hits = nullptr;
    uint32_t hits_cap = 0;
    uint32_t* d_dump_u = nullptr;
    uint32_t* d_dump_addr = nullptr;
    size_t dump_cap_keys = 0;
    uint32_t dump_lanes = 0, dump_keys = 0;  // of the last dumping launch
    uint32_t launch_max_hits = 0;            // largest max_hits since the last collect
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;
    bool initialised = false;
    fe tu[LXMFV_MAX_HALF_GROUP + 1], tv[LXMFV_MAX_HALF_GROUP + 1];  // grouped walk: J, 1Q .. MQ
    std::string err;
};

namespace {

int fail(lxmfv_handle* h, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    return code;
}

#define CU(h, call)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail((h), LXMFV_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                 \
    } while (0)

constexpr int minb(int block) { return block == 512 ? 1 : block == 256 ? 2 : 4; }

// The kernels for a configuration: block 128 runs without the phase barrier;
// 256 and 512 with or without it.  `low_regs` (LXMFV_FLAG_REGCAP_80): the
// G = 256, 256-thread, phase-barrier kernel built for three blocks per SM.
// DUMP: the build with the dump window's code, for launches that ask for one.
template <int M, bool DUMP>
const void* group_kernel_ptr_d(uint32_t block, bool sync, bool low_regs) {
    if (low_regs) {
        if constexpr (M == 128) {
            if (block == 256 && sync) return (const void*)lxk::group_walk_kernel<128, 256, 3, true, DUMP>;
        }
        return nullptr;
    }
    if (block == 128) return (const void*)lxk::group_walk_kernel<M, 128, minb(128), false, DUMP>;
    if (block == 256)
        return sync ? (const void*)lxk::group_walk_kernel<M, 256, minb(256), true, DUMP>
                    : (const void*)lxk::group_walk_kernel<M, 256, minb(256), false, DUMP>;
    if (block == 512)
        return sync ? (const void*)lxk::group_walk_kernel<M, 512, minb(512), true, DUMP>
                    : (const void*)lxk::group_walk_kernel<M, 512, minb(512), false, DUMP>;
    return nullptr;
}

template <int M>
const void* group_kernel_ptr(uint32_t block, bool sync, bool low_regs, bool dump) {
    return dump ? group_kernel_ptr_d<M, true>(block, sync, low_regs) : group_kernel_ptr_d<M, false>(block, sync, low_regs);
}

template <int B, bool DUMP>
const void* xadd_kernel_ptr_d(uint32_t block, bool sync, bool low_regs) {
    if (low_regs) return nullptr;
    if (block == 128) return (const void*)lxk::walk_kernel<B, 128, minb(128), false, DUMP>;
    if (block == 256)
        return sync ? (const void*)lxk::walk_kernel<B, 256, minb(256), true, DUMP>
                    : (const void*)lxk::walk_kernel<B, 256, minb(256), false, DUMP>;
    if (block == 512)
        return sync ? (const void*)lxk::walk_kernel<B, 512, minb(512), true, DUMP>
                    : (const void*)lxk::walk_kernel<B, 512, minb(512), false, DUMP>;
    return nullptr;
}

template <int B>
const void* xadd_kernel_ptr(uint32_t block, bool sync, bool low_regs, bool dump) {
    return dump ? xadd_kernel_ptr_d<B, true>(block, sync, low_regs) : xadd_kernel_ptr_d<B, false>(block, sync, low_regs);
}

// The warp-specialised grouped walk: 8 walker warps and 16 hash warps per
// block (768 threads, 256 lanes), 4 slots per walker warp's ring.  The block
// is launched at the kernel's register count (80 per thread: 61,440), and the
// roles then move to 128 registers (walkers: the field arithmetic with the
// next group's forward product) and 56 (hash warps): 256 x 128 + 512 x 56 =
// 61,440.  ws_regsplit_fits checks that sum against the built kernel before
// the first launch.
constexpr int kWsF = 8, kWsC = 2, kWsS = 4, kWsPRegs = 128, kWsQRegs = 56;
constexpr uint32_t kWsThreads = 32 * kWsF * (1 + kWsC);
constexpr uint32_t kWsLanesPerBlock = 32 * kWsF;
constexpr size_t kWsSmem = sizeof(lxk::WsShared<kWsF, kWsS>);

template <int M>
const void* ws_kernel_ptr(bool dump) {
    return dump ? (const void*)lxk::group_walk_ws_kernel<M, kWsF, kWsC, kWsS, true, kWsPRegs, kWsQRegs>
                : (const void*)lxk::group_walk_ws_kernel<M, kWsF, kWsC, kWsS, false, kWsPRegs, kWsQRegs>;
}

// Whether the register split fits the registers a block of the built kernel
// is launched with (setmaxnreg.inc waits for registers the other warps give
// back; a split above the launch total would wait for ever).
bool ws_regsplit_fits(const void* fn) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) return false;
    const long have = (long)fa.numRegs * kWsThreads;
    const long need = 32L * kWsF * kWsPRegs + 32L * kWsF * kWsC * kWsQRegs;
    return have >= need;
}

const void* ws_kernel_for(uint32_t batch, bool dump) {
    switch (batch) {
        case 512: return ws_kernel_ptr<256>(dump);
        case 1024: return ws_kernel_ptr<512>(dump);
    }
    return nullptr;
}

// The walk kernel of a configuration (null when unsupported).
const void* walk_kernel_ptr(uint32_t walk, uint32_t batch, uint32_t block, bool sync, bool low_regs,
                            bool dump = false) {
    if (walk == LXMFV_WALK_XADD) {
        switch (batch) {
            case 16: return xadd_kernel_ptr<16>(block, sync, low_regs, dump);
            case 32: return xadd_kernel_ptr<32>(block, sync, low_regs, dump);
            case 64: return xadd_kernel_ptr<64>(block, sync, low_regs, dump);
            case 128: return xadd_kernel_ptr<128>(block, sync, low_regs, dump);
        }
    } else if (walk == LXMFV_WALK_GROUP) {
        switch (batch) {
            case 32: return group_kernel_ptr<16>(block, sync, low_regs, dump);
            case 64: return group_kernel_ptr<32>(block, sync, low_regs, dump);
            case 128: return group_kernel_ptr<64>(block, sync, low_regs, dump);
            case 256: return group_kernel_ptr<128>(block, sync, low_regs, dump);
            case 512: return group_kernel_ptr<256>(block, sync, low_regs, dump);
            case 1024: return group_kernel_ptr<512>(block, sync, low_regs, dump);
        }
    }
    return nullptr;
}

template <int B>
void launch_xadd(lxmfv_handle* h, const lxk::WalkArgs& wa) {
    const unsigned grid = (h->lanes + h->block - 1) / h->block;
    typedef void (*fn_t)(lxk::WalkArgs);
    const fn_t fn = (fn_t)xadd_kernel_ptr<B>(h->block, h->sync, h->low_regs, wa.em.dump_lanes > 0);
    fn<<<grid, h->block, 0, h->stream>>>(wa);
}

template <int M>
void launch_group_ws(lxmfv_handle* h, const lxk::EmitArgs& em, uint32_t iters) {
    if constexpr (M == 256 || M == 512) {
        lxk::WsArgs<M> a;
        a.g.state = h->d_state;
        a.g.ns = h->d_ns;
        a.g.lanes = h->lanes;
        a.g.iters = iters;
        a.g.em = em;
        if constexpr (M <= 256) {
            for (int i = 0; i <= M; i++) {
                a.g.t.u[i] = h->tu[i];
                a.g.t.v[i] = h->tv[i];
            }
        }
        a.err = h->d_err;
        const unsigned grid = (h->lanes + kWsLanesPerBlock - 1) / kWsLanesPerBlock;
        typedef void (*fn_t)(lxk::WsArgs<M>);
        const fn_t fn = (fn_t)ws_kernel_ptr<M>(em.dump_lanes > 0);
        fn<<<grid, kWsThreads, kWsSmem, h->stream>>>(a);
    }
}

template <int M>
void launch_group(lxmfv_handle* h, const lxk::EmitArgs& em, uint32_t iters) {
    lxk::GroupArgsFor<M> ga;
    ga.state = h->d_state;
    ga.ns = h->d_ns;
    ga.lanes = h->lanes;
    ga.iters = iters;
    ga.em = em;
    if constexpr (M <= 256) {
        for (int i = 0; i <= M; i++) {
            ga.t.u[i] = h->tu[i];
            ga.t.v[i] = h->tv[i];
        }
    }
    const unsigned grid = (h->lanes + h->block - 1) / h->block;
    typedef void (*fn_t)(lxk::GroupArgsFor<M>);
    const fn_t fn = (fn_t)group_kernel_ptr<M>(h->block, h->sync, h->low_regs, em.dump_lanes > 0);
    fn<<<grid, h->block, 0, h->stream>>>(ga);
}

void launch_walk(lxmfv_handle* h, const lxk::EmitArgs& em, uint32_t iters, const fe& q) {
    if (h->walk == LXMFV_WALK_XADD) {
        lxk::WalkArgs wa;
        memset(&wa, 0, sizeof wa);
        wa.state = h->d_state;
        wa.ns = h->d_ns;
        wa.lanes = h->lanes;
        wa.iters = iters;
        wa.q = q;
        wa.em = em;
        switch (h->batch) {
            case 16: launch_xadd<16>(h, wa); break;
            case 32: launch_xadd<32>(h, wa); break;
            case 64: launch_xadd<64>(h, wa); break;
            default: launch_xadd<128>(h, wa); break;
        }
    } else if (h->ws) {
        if (h->batch == 512)
            launch_group_ws<256>(h, em, iters);
        else
            launch_group_ws<512>(h, em, iters);
    } else {
        switch (h->batch) {
            case 32: launch_group<16>(h, em, iters); break;
            case 64: launch_group<32>(h, em, iters); break;
            case 128: launch_group<64>(h, em, iters); break;
            case 256: launch_group<128>(h, em, iters); break;
            case 512: launch_group<256>(h, em, iters); break;
            default: launch_group<512>(h, em, iters); break;
        }
    }
}

void fill_addr_consts(lxsha::AddrConsts& ac, const uint32_t ed[8], const uint32_t nh[3], const uint32_t want[4],
                      const uint32_t mask[4]) {
    ac.one = 1;
    for (int i = 0; i < 8; i++) ac.ed[i] = ed ? ed[i] : 0;
    for (int i = 0; i < 3; i++) ac.nh[i] = nh[i];
    for (int i = 0; i < 4; i++) {
        ac.want[i] = want ? want[i] : 0;
        ac.mask[i] = mask ? mask[i] : 0;
    }
}

int ensure_hits(lxmfv_handle* h, uint32_t cap) {
    if (cap <= h->hits_cap) return LXMFV_OK;
    // Grow only between launches: every queued launch has finished here.
    CU(h, cudaStreamSynchronize(h->stream));
    lxk::Hit* nh = nullptr;
    CU(h, cudaMalloc(&nh, sizeof(lxk::Hit) * cap));
    if (h->d_hits) {
        CU(h, cudaMemcpyAsync(nh, h->d_hits, sizeof(lxk::Hit) * h->hits_cap, cudaMemcpyDeviceToDevice, h->stream));
        CU(h, cudaStreamSynchronize(h->stream));
        cudaFree(h->d_hits);
    }
    h->d_hits = nh;
    h->hits_cap = cap;
    return LXMFV_OK;
}

int ensure_dump(lxmfv_handle* h, size_t keys) {
    if (keys <= h->dump_cap_keys) return LXMFV_OK;
    CU(h, cudaStreamSynchronize(h->stream));
    cudaFree(h->d_dump_u);
    cudaFree(h->d_dump_addr);
    h->d_dump_u = nullptr;
    h->d_dump_addr = nullptr;
    h->dump_cap_keys = 0;
    CU(h, cudaMalloc(&h->d_dump_u, keys * 8 * sizeof(uint32_t)));
    CU(h, cudaMalloc(&h->d_dump_addr, keys * 4 * sizeof(uint32_t)));
    h->dump_cap_keys = keys;
    return LXMFV_OK;
}

int set_device(lxmfv_handle* h) {
    CU(h, cudaSetDevice(h->device));
    return LXMFV_OK;
}

fe words8(const uint32_t w[8]) {
    fe x;
    for (int i = 0; i < 8; i++) x.v[i] = w[i];
    return x;
}

// u(8B), the fixed step point (mod.rs:111, main.rs:244), as 8 LE words.
fe u8b() {
    static const uint32_t U8B[8] = {0x48c99968u, 0xf1716fedu, 0xad74a91eu, 0x7a78edcau,
                                    0xc8b65ca1u, 0xd83b884du, 0xaad65c2du, 0x275fa6d7u};
    return words8(U8B);
}

// v(8B): the even square root of u^3 + A u^2 + u at u = u(8B); the grouped
// walk's points are all multiples of this Q.  And its negation, p - v.
fe v8b() {
    static const uint32_t V[8] = {0x9f728718u, 0xc5296d6eu, 0x70c591f9u, 0x4f479c67u,
                                  0x4066b08cu, 0x8dcf4469u, 0x8fb939e4u, 0x6085bbbau};
    return words8(V);
}

fe v8b_neg() {
    static const uint32_t V[8] = {0x608d78d5u, 0x3ad69291u, 0x8f3a6e06u, 0xb0b86398u,
                                  0xbf994f73u, 0x7230bb96u, 0x7046c61bu, 0x1f7a4445u};
    return words8(V);
}

int check_scalars(lxmfv_handle* h, const uint8_t* scalars, size_t count) {
    for (size_t t = 0; t < count; t++) {
        const uint8_t* k = scalars + 32 * t;
        if ((k[0] & 7) != 0 || (k[31] & 0xC0) != 0x40)
            return fail(h, LXMFV_ERR_ARG, "scalar %zu is not clamped (k mod 8 = 0, bit 254 set, bit 255 clear)", t);
        bool low_all_clear = k[31] == 64;
        for (int i = 0; i < 31; i++) low_all_clear = low_all_clear && k[i] == 0;
        if (low_all_clear) return fail(h, LXMFV_ERR_ARG, "scalar %zu is 2^254: k - 8 would not be clamped", t);
    }
    return LXMFV_OK;
}

// The grouped walk's table, computed once on the device and kept on the host
// to travel in every launch's parameter block.
int build_group_table(lxmfv_handle* h) {
    const uint32_t m = h->batch / 2;
    fe *du = nullptr, *dv = nullptr;
    cudaError_t e = cudaMalloc(&du, sizeof(fe) * (m + 1));
    if (e == cudaSuccess) e = cudaMalloc(&dv, sizeof(fe) * (m + 1));
    if (e == cudaSuccess) {
        lxk::group_table_kernel<<<1, ((m + 1 + 31) / 32) * 32, 0, h->stream>>>(du, dv, m, u8b(), v8b());
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->tu, du, sizeof(fe) * (m + 1), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->tv, dv, sizeof(fe) * (m + 1), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(du);
    cudaFree(dv);
    if (e == cudaSuccess && m > 256) {
        // The G = 1024 kernels read the table from constant memory.  Every
        // handle on the device writes the same bytes, so a launch of another
        // handle that reads it meanwhile sees no change.
        e = cudaMemcpyToSymbolAsync(lxk::c_group_u, h->tu, sizeof(fe) * (m + 1), 0, cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyToSymbolAsync(lxk::c_group_v, h->tv, sizeof(fe) * (m + 1), 0, cudaMemcpyHostToDevice,
                                        h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    if (e != cudaSuccess) return fail(h, LXMFV_ERR_CUDA, "group table: %s", cudaGetErrorString(e));
    return LXMFV_OK;
}

}  // namespace

extern "C" {

int lxmfv_open(const lxmfv_options* opts, lxmfv_handle** out) {
    if (!out) return LXMFV_ERR_ARG;
    *out = nullptr;
    lxmfv_handle* h = new (std::nothrow) lxmfv_handle();
    if (!h) return LXMFV_ERR_NOMEM;
    *out = h;
    lxmfv_options o{};
    if (opts) o = *opts;
    h->device = o.device;
    h->walk = o.walk;
    // 0: the fastest keys per inversion of each walk (the autotuner's choice).
    h->batch = o.batch ? o.batch : (o.walk == LXMFV_WALK_XADD ? 128 : 1024);
    // Default launch shape (block 0): 512 threads with the phase barrier, the
    // fastest measured on B200 for both walks; otherwise the flags decide.
    h->block = o.block ? o.block : 512;
    h->sync = o.block ? (o.flags & LXMFV_FLAG_PHASE_SYNC) != 0 : true;
    h->low_regs = (o.flags & LXMFV_FLAG_REGCAP_80) != 0;
    h->ws = (o.flags & LXMFV_FLAG_WARP_SPEC) != 0;
    if (h->ws && (h->walk != LXMFV_WALK_GROUP || !ws_kernel_for(h->batch, false) || h->low_regs ||
                  (o.block && o.block != kWsThreads)))
        return fail(h, LXMFV_ERR_ARG, "LXMFV_FLAG_WARP_SPEC needs the grouped walk, batch 512 or 1024 and block 0 or %u",
                    kWsThreads);
    if (h->ws) h->block = kWsThreads;
    if (h->walk != LXMFV_WALK_GROUP && h->walk != LXMFV_WALK_XADD)
        return fail(h, LXMFV_ERR_ARG, "walk %u: 0 grouped, 1 x-only", h->walk);
    if (h->low_regs && !walk_kernel_ptr(h->walk, h->batch, h->block, h->sync, true))
        return fail(h, LXMFV_ERR_ARG,
                    "LXMFV_FLAG_REGCAP_80 needs the grouped walk, batch 256, block 256 and LXMFV_FLAG_PHASE_SYNC");
    if (!h->ws && !walk_kernel_ptr(h->walk, h->batch, h->block, h->sync, h->low_regs))
        return fail(h, LXMFV_ERR_ARG,
                    "unsupported batch %u / block %u (x-only walk: batch 16, 32, 64, 128; grouped walk: "
                    "batch 32, 64, 128, 256, 512, 1024; block 128, 256 or 512)",
                    h->batch, h->block);
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(h, LXMFV_ERR_CUDA, "no CUDA device: %s", e != cudaSuccess ? cudaGetErrorString(e) : "none found");
    if (h->device < 0 || h->device >= count)
        return fail(h, LXMFV_ERR_ARG, "device %d out of range (%d devices)", h->device, count);
    if (int rc = set_device(h)) return rc;
    cudaDeviceProp prop;
    CU(h, cudaGetDeviceProperties(&prop, h->device));
    h->sms = prop.multiProcessorCount;
    h->cc_major = prop.major;
    h->cc_minor = prop.minor;
    h->name = prop.name;
    if (prop.major != 10 || prop.minor != 0)
        return fail(h, LXMFV_ERR_CUDA, "%s is compute %d.%d; this library is built for sm_100a (B200) only", prop.name,
                    prop.major, prop.minor);
    if (o.stream) {
        h->stream = (cudaStream_t)o.stream;
    } else {
        CU(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->own_stream = true;
    }
    CU(h, cudaEventCreate(&h->ev0));
    CU(h, cudaEventCreate(&h->ev1));
    int per_sm = 0;
    if (h->ws) {
        // The ring buffers take more than the default 48 KB of dynamic shared memory.
        for (int dump = 0; dump < 2; dump++) {
            if (!ws_regsplit_fits(ws_kernel_for(h->batch, dump != 0)))
                return fail(h, LXMFV_ERR_STATE, "warp-specialised walk: the register split exceeds the launch registers");
            CU(h, cudaFuncSetAttribute(ws_kernel_for(h->batch, dump != 0), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kWsSmem));
        }
        CU(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ws_kernel_for(h->batch, false), (int)h->block,
                                                            kWsSmem));
        if (per_sm < 1) return fail(h, LXMFV_ERR_CUDA, "warp-specialised walk cannot be resident (batch %u)", h->batch);
        h->lanes = o.lanes ? o.lanes : (uint32_t)(h->sms * per_sm) * kWsLanesPerBlock;
        CU(h, cudaMalloc(&h->d_err, sizeof(uint32_t)));
        CU(h, cudaMemsetAsync(h->d_err, 0, sizeof(uint32_t), h->stream));
    } else {
        CU(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                  &per_sm, walk_kernel_ptr(h->walk, h->batch, h->block, h->sync, h->low_regs), (int)h->block, 0));
        if (per_sm < 1)
            return fail(h, LXMFV_ERR_CUDA, "walk kernel cannot be resident (batch %u, block %u)", h->batch, h->block);
        h->lanes = o.lanes ? o.lanes : (uint32_t)(h->sms * per_sm) * h->block;
    }
    CU(h, cudaMalloc(&h->d_state, (size_t)h->lanes * 32 * sizeof(uint32_t)));
    CU(h, cudaMalloc(&h->d_ns, (size_t)h->lanes * sizeof(uint64_t)));
    CU(h, cudaMalloc(&h->d_hit_count, sizeof(uint32_t)));
    CU(h, cudaMemsetAsync(h->d_hit_count, 0, sizeof(uint32_t), h->stream));
    CU(h, cudaMemsetAsync(h->d_state, 0, (size_t)h->lanes * 32 * sizeof(uint32_t), h->stream));
    CU(h, cudaMemsetAsync(h->d_ns, 0, (size_t)h->lanes * sizeof(uint64_t), h->stream));
    if (int rc = ensure_hits(h, 4096)) return rc;
    if (h->walk == LXMFV_WALK_GROUP)
        if (int rc = build_group_table(h)) return rc;
    CU(h, cudaStreamSynchronize(h->stream));
    h->err.clear();
    return LXMFV_OK;
}

const char* lxmfv_last_error(const lxmfv_handle* h) { return h ? h->err.c_str() : "null handle"; }

int lxmfv_describe(const lxmfv_handle* h, char* buf, size_t len) {
    if (!h) return LXMFV_ERR_ARG;
    return snprintf(buf, len, "%s (CUDA, compute %d.%d, %d SMs)", h->name.c_str(), h->cc_major, h->cc_minor, h->sms);
}

uint32_t lxmfv_threads(const lxmfv_handle* h) { return h ? h->lanes : 0; }

uint64_t lxmfv_batch(const lxmfv_handle* h) { return h ? h->batch : 0; }

uint32_t lxmfv_walk(const lxmfv_handle* h) { return h ? h->walk : 0; }

int lxmfv_init(lxmfv_handle* h, const uint32_t* u_prev_cur, size_t n_words) {
    if (!h || !u_prev_cur) return fail(h, LXMFV_ERR_ARG, "null argument");
    if (!h->d_state) return fail(h, LXMFV_ERR_STATE, "handle is not open");
    if (n_words != (size_t)h->lanes * 16)
        return fail(h, LXMFV_ERR_ARG, "u_prev_cur has %zu words; %u lanes need %zu", n_words, h->lanes,
                    (size_t)h->lanes * 16);
    if (int rc = set_device(h)) return rc;
    uint32_t* d = nullptr;
    CU(h, cudaMalloc(&d, n_words * sizeof(uint32_t)));
    cudaError_t e = cudaMemcpyAsync(d, u_prev_cur, n_words * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        if (h->walk == LXMFV_WALK_XADD) {
            lxk::init_kernel<<<(h->lanes + 255) / 256, 256, 0, h->stream>>>(h->d_state, h->d_ns, d, h->lanes);
        } else {
            const uint32_t m = h->batch / 2;
            lxk::group_init_kernel<<<(h->lanes + 127) / 128, 128, 0, h->stream>>>(h->d_state, h->d_ns, d, h->lanes,
                                                                                   u8b(), v8b_neg(), h->tu[m], h->tv[m]);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(h, LXMFV_ERR_CUDA, "init: %s", cudaGetErrorString(e));
    h->initialised = true;
    h->err.clear();
    return LXMFV_OK;
}

int lxmfv_init_from_scalars(lxmfv_handle* h, const uint8_t* scalars, size_t n_bytes) {
    if (!h || !scalars) return fail(h, LXMFV_ERR_ARG, "null argument");
    if (!h->d_state) return fail(h, LXMFV_ERR_STATE, "handle is not open");
    if (n_bytes != (size_t)h->lanes * 32)
        return fail(h, LXMFV_ERR_ARG, "scalars have %zu bytes; %u lanes need %zu", n_bytes, h->lanes,
                    (size_t)h->lanes * 32);
    if (int rc = check_scalars(h, scalars, h->lanes)) return rc;
    if (int rc = set_device(h)) return rc;
    uint32_t* d = nullptr;
    CU(h, cudaMalloc(&d, n_bytes));
    cudaError_t e = cudaMemcpyAsync(d, scalars, n_bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        if (h->walk == LXMFV_WALK_XADD) {
            lxk::ladder_kernel<<<(h->lanes + 127) / 128, 128, 0, h->stream>>>(h->d_state, h->d_ns, d, h->lanes, u8b());
        } else {
            lxk::group_start_kernel<<<(h->lanes + 127) / 128, 128, 0, h->stream>>>(h->d_state, h->d_ns, d, h->lanes,
                                                                                    h->batch / 2, u8b(), v8b());
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(h, LXMFV_ERR_CUDA, "init_from_scalars: %s", cudaGetErrorString(e));
    h->initialised = true;
    h->err.clear();
    return LXMFV_OK;
}

int lxmfv_first_public_keys(lxmfv_handle* h, const uint8_t* scalars, size_t count, uint32_t* u_prev_cur) {
    if (!h || !scalars || !u_prev_cur) return fail(h, LXMFV_ERR_ARG, "null argument");
    if (!h->sms) return fail(h, LXMFV_ERR_STATE, "handle is not open");
    if (count == 0) return LXMFV_OK;
    if (count > (1u << 30)) return fail(h, LXMFV_ERR_ARG, "count %zu too large", count);
    if (int rc = check_scalars(h, scalars, count)) return rc;
    if (int rc = set_device(h)) return rc;
    uint32_t *ds = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&ds, count * 32);
    if (e == cudaSuccess) e = cudaMalloc(&dout, count * 64);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds, scalars, count * 32, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        lxk::first_keys_kernel<<<(unsigned)((count + 127) / 128), 128, 0, h->stream>>>(dout, ds, (uint32_t)count, u8b());
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(u_prev_cur, dout, count * 64, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(ds);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(h, LXMFV_ERR_CUDA, "first_public_keys: %s", cudaGetErrorString(e));
    h->err.clear();
    return LXMFV_OK;
}

int lxmfv_launch_async(lxmfv_handle* h, const lxmfv_launch_args* args) {
    if (!h || !args) return fail(h, LXMFV_ERR_ARG, "null argument");
    if (!h->initialised) return fail(h, LXMFV_ERR_STATE, "launch before init");
    if (args->iters == 0) return fail(h, LXMFV_ERR_ARG, "iters must be at least 1");
    // The warp-specialised walk counts its ring's hand-overs (iters x (M + 1)) in 32 bits.
    if (h->ws && (uint64_t)args->iters * (h->batch / 2 + 1) >= (1ull << 32))
        return fail(h, LXMFV_ERR_ARG, "iters %u too large for the warp-specialised walk", args->iters);
    if (int rc = set_device(h)) return rc;
    // The step point is fixed: both walks' tables and start points are built
    // from u(8B), so a launch must use it too (the reference passes it per
    // launch, mod.rs:111).
    fe q = u8b();
    for (int i = 0; i < 8; i++)
        if (args->q[i] != q.v[i]) return fail(h, LXMFV_ERR_ARG, "q must be u(8B), the walk's step point");
    lxk::EmitArgs em;
    memset(&em, 0, sizeof em);
    fill_addr_consts(em.ac, args->ed, args->name_hash, args->want, args->mask);
    if (int rc = ensure_hits(h, std::max<uint32_t>(args->max_hits, 1))) return rc;
    em.hit_count = h->d_hit_count;
    em.hits = h->d_hits;
    em.max_hits = args->max_hits;
    h->launch_max_hits = std::max(h->launch_max_hits, args->max_hits);
    if (args->dump_threads > 0) {
        const uint32_t dl = std::min(args->dump_threads, h->lanes);
        const uint32_t dk = args->dump_keys ? args->dump_keys : h->batch;
        if ((uint64_t)dk > (uint64_t)args->iters * h->batch)
            return fail(h, LXMFV_ERR_ARG, "dump_keys %u exceeds the %llu keys a lane walks in this launch", dk,
                        (unsigned long long)args->iters * h->batch);
        if (int rc = ensure_dump(h, (size_t)dl * dk)) return rc;
        em.dump_lanes = dl;
        em.dump_keys = dk;
        em.dump_u = h->d_dump_u;
        em.dump_addr = h->d_dump_addr;
        h->dump_lanes = dl;
        h->dump_keys = dk;
    }
    CU(h, cudaEventRecord(h->ev0, h->stream));
    launch_walk(h, em, args->iters, q);
    CU(h, cudaGetLastError());
    CU(h, cudaEventRecord(h->ev1, h->stream));
    h->timed = true;
    h->err.clear();
    return LXMFV_OK;
}

int lxmfv_collect(lxmfv_handle* h, lxmfv_hit* hits, uint32_t hits_cap, uint32_t* n_hits, uint32_t* dump,
                  uint32_t* dump_addr) {
    if (!h || !n_hits) return fail(h, LXMFV_ERR_ARG, "null argument");
    if (int rc = set_device(h)) return rc;
    CU(h, cudaStreamSynchronize(h->stream));
    uint32_t count = 0;
    CU(h, cudaMemcpy(&count, h->d_hit_count, sizeof count, cudaMemcpyDeviceToHost));
    const uint32_t stored = std::min(std::min(count, h->launch_max_hits), h->hits_cap);
    const uint32_t give = hits ? std::min(stored, hits_cap) : 0;
    if (give > 0) CU(h, cudaMemcpy(hits, h->d_hits, sizeof(lxk::Hit) * give, cudaMemcpyDeviceToHost));
    const size_t dumped = (size_t)h->dump_lanes * h->dump_keys;
    if (dump && dumped) CU(h, cudaMemcpy(dump, h->d_dump_u, dumped * 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (dump_addr && dumped)
        CU(h, cudaMemcpy(dump_addr, h->d_dump_addr, dumped * 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    CU(h, cudaMemsetAsync(h->d_hit_count, 0, sizeof(uint32_t), h->stream));
    uint32_t gave_up = 0;
    if (h->d_err) {
        CU(h, cudaMemcpy(&gave_up, h->d_err, sizeof gave_up, cudaMemcpyDeviceToHost));
        CU(h, cudaMemsetAsync(h->d_err, 0, sizeof(uint32_t), h->stream));
    }
    CU(h, cudaStreamSynchronize(h->stream));
    h->launch_max_hits = 0;
    if (gave_up) {
        // Some lanes stopped part-way: their state no longer matches their walk index.
        h->initialised = false;
        h->dump_lanes = 0;
        h->dump_keys = 0;
        return fail(h, LXMFV_ERR_CUDA, "a warp-specialised launch gave up waiting on its ring; initialise again");
    }
    h->dump_lanes = 0;
    h->dump_keys = 0;
    *n_hits = count;
    h->err.clear();
    return LXMFV_OK;
}

int lxmfv_launch(lxmfv_handle* h, const lxmfv_launch_args* args, lxmfv_hit* hits, uint32_t hits_cap,
                 uint32_t* n_hits, uint32_t* dump, uint32_t* dump_addr) {
    if (int rc = lxmfv_launch_async(h, args)) return rc;
    return lxmfv_collect(h, hits, hits_cap, n_hits, dump, dump_addr);
}

float lxmfv_last_kernel_ms(const lxmfv_handle* h) {
    if (!h || !h->timed) return -1.0f;
    float ms = -1.0f;
    if (cudaEventSynchronize(h->ev1) != cudaSuccess) return -1.0f;
    if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) != cudaSuccess) return -1.0f;
    return ms;
}

void lxmfv_close(lxmfv_handle* h) {
    if (!h) return;
    if (h->sms) {
        cudaSetDevice(h->device);
        if (h->stream) cudaStreamSynchronize(h->stream);
        cudaFree(h->d_state);
        cudaFree(h->d_ns);
        cudaFree(h->d_hit_count);
        cudaFree(h->d_hits);
        cudaFree(h->d_dump_u);
        cudaFree(h->d_dump_addr);
        cudaFree(h->d_err);
        if (h->ev0) cudaEventDestroy(h->ev0);
        if (h->ev1) cudaEventDestroy(h->ev1);
        if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    }
    delete h;
}

// ---- Primitive kernels.

int lxmfv_fe_op(lxmfv_handle* h, int op, const uint32_t* a, const uint32_t* b, uint32_t* out, uint64_t count,
                uint32_t group) {
    if (!h || !a || !out || (op == 0 && !b)) return fail(h, LXMFV_ERR_ARG, "null argument");
    if (op < 0 || op > 3) return fail(h, LXMFV_ERR_ARG, "op %d: 0 mul, 1 square, 2 invert, 3 batch invert", op);
    if (op == 3 && (group < 1 || group > 256)) return fail(h, LXMFV_ERR_ARG, "group %u not in 1..256", group);
    if (count == 0) return LXMFV_OK;
    if (int rc = set_device(h)) return rc;
    const size_t bytes = count * 8 * sizeof(uint32_t);
    uint32_t *da = nullptr, *db = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&da, bytes);
    if (e == cudaSuccess && op == 0) e = cudaMalloc(&db, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&dout, bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(da, a, bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && op == 0) e = cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        const int grid = h->sms * 8;
        if (op == 3) {
            lxk::fe_batch_invert_kernel<<<grid, 128, 0, h->stream>>>(da, dout, count, group);
        } else {
            lxk::fe_op_kernel<<<grid, 256, 0, h->stream>>>(op, da, db, dout, count);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(da);
    cudaFree(db);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(h, LXMFV_ERR_CUDA, "fe_op: %s", cudaGetErrorString(e));
    return LXMFV_OK;
}

int lxmfv_address_chain(lxmfv_handle* h, const uint8_t* pks, const uint8_t name_hash[10], uint8_t* out,
                        uint64_t count) {
    if (!h || !pks || !name_hash || !out) return fail(h, LXMFV_ERR_ARG, "null argument");
    if (count == 0) return LXMFV_OK;
    if (int rc = set_device(h)) return rc;
    uint32_t nh[3] = {(uint32_t)name_hash[0] << 24 | (uint32_t)name_hash[1] << 16 | (uint32_t)name_hash[2] << 8 | name_hash[3],
                      (uint32_t)name_hash[4] << 24 | (uint32_t)name_hash[5] << 16 | (uint32_t)name_hash[6] << 8 | name_hash[7],
                      (uint32_t)name_hash[8] << 24 | (uint32_t)name_hash[9] << 16};
    lxsha::AddrConsts ac;
    fill_addr_consts(ac, nullptr, nh, nullptr, nullptr);
    uint32_t *dpk = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&dpk, count * 64);
    if (e == cudaSuccess) e = cudaMalloc(&dout, count * 16);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dpk, pks, count * 64, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        lxk::address_chain_kernel<<<h->sms * 8, 256, 0, h->stream>>>(dpk, ac, dout, count);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, count * 16, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dpk);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(h, LXMFV_ERR_CUDA, "address_chain: %s", cudaGetErrorString(e));
    return LXMFV_OK;
}

int lxmfv_peak_probe(lxmfv_handle* h, int kind, float ms, double* ops_per_s) {
    if (!h || !ops_per_s || kind < 0 || kind > 7) return fail(h, LXMFV_ERR_ARG, "bad argument");
    if (int rc = set_device(h)) return rc;
    uint32_t* sink = nullptr;
    CU(h, cudaMalloc(&sink, sizeof(uint32_t)));
    const int blocks = h->sms * 8, threads = 256;
    const double per_iter = (double)blocks * threads * 16 * 8 * ((kind == 2 || kind == 5) ? 2 : 1);
    uint32_t iters = 64;
    float t = 0;
    cudaError_t e = cudaSuccess;
    for (int pass = 0; pass < 4 && e == cudaSuccess; pass++) {
        e = cudaEventRecord(h->ev0, h->stream);
        if (e == cudaSuccess) {
            lxk::probe_kernel<<<blocks, threads, 0, h->stream>>>(kind, iters, 12345u + pass, sink);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaEventRecord(h->ev1, h->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(h->ev1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, h->ev0, h->ev1);
        if (e != cudaSuccess) break;
        if (pass < 3 && t > 0) {
            const double want = std::max(ms, 1.0f);
            iters = (uint32_t)std::min(1e7, std::max(1.0, iters * want / t));
        }
    }
    cudaFree(sink);
    if (e != cudaSuccess) return fail(h, LXMFV_ERR_CUDA, "peak_probe: %s", cudaGetErrorString(e));
    *ops_per_s = per_iter * iters / (t * 1e-3);
    return LXMFV_OK;
}

}  // extern "C"
