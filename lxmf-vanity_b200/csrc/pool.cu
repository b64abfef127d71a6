// The search pool: many independent searches (each its own prefix, aspect
// and identity) walked by one persistent kernel.
//
// The reference runs one search per process (GpuSearch, src/gpu/mod.rs:86-174)
// and scales out by starting more processes (fleet.sh).  Here a pool of
// walker lanes lives on the device for the pool's lifetime; searches are
// admitted into it (lxmfv_pool_submit), walked together, and retired
// (lxmfv_pool_retire) as their hits arrive, freeing lanes for the next ones.
//
// Device layout:
//   - lanes in chunks of 32 (one warp).  A chunk belongs to one search, so a
//     warp's prefix, aspect and Ed25519 key are uniform and a mixed batch of
//     searches does not diverge;
//   - lane state as in the grouped walk (u_C, v_C word-major, walk index);
//   - a search table (the hash chain's constants per search slot);
//   - the work queue: the active chunks, in search order.  Each step, the
//     persistent kernel's blocks (one per SM, 16 warps) take items of 16
//     chunks from it with an atomic counter until it is empty, and walk every
//     lane of an item `groups` groups, so every active lane advances by the
//     same number of keys per step: a search's hits do not depend on what
//     else is in the pool;
//   - a hit queue of (search, lane within the search, walk index).
// One step is a CUDA graph, captured once per `groups`: reset the work
// counter, run the persistent kernel, copy the hit count and hits to pinned
// host memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/lxmfv.h"
#include "group_kernels.cuh"

namespace lxk {

struct PoolSearch {
    lxsha::AddrConsts ac;
};

struct PoolHit {
    uint32_t search;
    uint32_t lane;  // lane index within the search
    uint64_t n;
};

constexpr int kPoolWarps = 16;  // warps per block (512 threads)

// The pool's group table: in the parameters up to M = 256, in constant
// memory (c_group_u / c_group_v, written at lxmfv_pool_open) at M = 512.
struct NoTable {};
template <int M>
using PoolTableFor = typename std::conditional<(M > 256), NoTable, GroupTable<M>>::type;
template <int M>
__device__ __forceinline__ const GroupTable<M>& pool_table(const GroupTable<M>& t) { return t; }
__device__ __forceinline__ ConstGroupTable pool_table(const NoTable&) { return ConstGroupTable{}; }

template <int M>
struct PoolArgs {
    uint32_t* state;               // [16][capacity]: u_C, v_C
    uint64_t* ns;                  // [capacity]
    uint32_t capacity;
    const uint32_t* queue;         // active chunk ids
    const uint32_t* n_queue;       // queue length (device scalar)
    const uint32_t* chunk_search;  // [capacity / 32] search slot of each chunk
    const uint32_t* chunk_first;   // [capacity / 32] index in its search of the chunk's first lane
    const PoolSearch* searches;
    uint32_t* head;                // work counter, zero at the start of a step
    uint32_t groups;               // groups per lane per step
    uint32_t* hit_count;
    PoolHit* hits;
    uint32_t max_hits;
    uint32_t one;                  // 1: the SHA-256 sums' multiplier (see madd)
    PoolTableFor<M> t;
};

struct PoolEmit {
    const lxsha::AddrConsts& ac;   // shared memory: this warp's search
    uint32_t* hit_count;
    PoolHit* hits;
    uint32_t max_hits;
    uint32_t search;
    uint32_t lane_in_search;
    bool active;
    uint32_t one;  // from the kernel parameters
    __device__ __forceinline__ void operator()(const fe& u, uint64_t key) const {
        uint32_t d[4];
        lxsha::dest_hash_one(u.v, ac.ed, ac, one, d);
        const bool match = ((d[0] & ac.mask[0]) == ac.want[0]) & ((d[1] & ac.mask[1]) == ac.want[1]) &
                           ((d[2] & ac.mask[2]) == ac.want[2]) & ((d[3] & ac.mask[3]) == ac.want[3]);
        if (active && match) {
            const uint32_t slot = atomicAdd(hit_count, 1u);
            if (slot < max_hits) {
                hits[slot].search = search;
                hits[slot].lane = lane_in_search;
                hits[slot].n = key;
            }
        }
    }
};

template <int M>
static __global__ void __launch_bounds__(32 * kPoolWarps, 1) pool_walk_kernel(const __grid_constant__ PoolArgs<M> a) {
    __shared__ uint32_t s_item;
    __shared__ lxsha::AddrConsts s_ac[kPoolWarps];
    const uint32_t warp = threadIdx.x >> 5, lid = threadIdx.x & 31;
    const uint32_t nq = *a.n_queue;
    const uint32_t n_items = (nq + kPoolWarps - 1) / kPoolWarps;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(a.head, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= n_items) break;  // the same for every thread of the block
        const uint32_t qi = item * kPoolWarps + warp;
        const bool active = qi < nq;  // a short last item: spare warps walk a copy and write nothing
        const uint32_t chunk = a.queue[active ? qi : nq - 1];
        const uint32_t search = a.chunk_search[chunk];
        constexpr int kWords = sizeof(lxsha::AddrConsts) / 4;
        if (lid < kWords)
            reinterpret_cast<uint32_t*>(&s_ac[warp])[lid] = reinterpret_cast<const uint32_t*>(&a.searches[search].ac)[lid];
        __syncwarp();
        const uint32_t lane = chunk * 32 + lid;
        fe uc = load_fe(a.state, 0, lane, a.capacity);
        fe vc = load_fe(a.state, 1, lane, a.capacity);
        uint64_t n = a.ns[lane];
        const PoolEmit emit{s_ac[warp], a.hit_count, a.hits, a.max_hits, search, a.chunk_first[chunk] + lid, active, a.one};
        walk_groups<M, true>(uc, vc, n, a.groups, pool_table(a.t), emit);
        if (active) {
            store_fe(a.state, 0, lane, a.capacity, uc);
            store_fe(a.state, 1, lane, a.capacity, vc);
            a.ns[lane] = n;
        }
        __syncthreads();  // s_item and s_ac are rewritten next
    }
}

// Start centres for `count` lanes of one search: lane i (a pool lane from
// lane_map) from start scalar i, C = (k/8 + M) Q as in group_start_kernel.
static __global__ void __launch_bounds__(128) pool_start_kernel(uint32_t* state, uint64_t* ns, uint32_t capacity,
                                                                 const uint32_t* __restrict__ scalars,
                                                                 const uint32_t* __restrict__ lane_map, uint32_t count,
                                                                 uint32_t m, fe q, fe vq) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint32_t s[8];
    scalar_over_8(scalars, i, (int)m, s);
    fe x2, z2, x3, z3, X, Y, Z, u, v;
    ladder(s, 253, q, x2, z2, x3, z3);
    recover_y(q, vq, x2, z2, x3, z3, X, Y, Z);
    to_affine(X, Y, Z, u, v);
    const uint32_t lane = lane_map[i];
    store_fe(state, 0, lane, capacity, u);
    store_fe(state, 1, lane, capacity, v);
    ns[lane] = 0;
}

}  // namespace lxk

struct lxmfv_pool {
    struct Search {
        bool active = false;
        uint32_t lanes = 0;
        std::vector<uint32_t> chunks;
        uint64_t keys_per_lane = 0;  // walk index every lane of the search has reached
    };
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t batch = 256, m = 128;
    uint32_t capacity = 0, chunks = 0, max_searches = 0, max_hits = 0;
    uint32_t* d_state = nullptr;
    uint64_t* d_ns = nullptr;
    uint32_t *d_queue = nullptr, *d_nq = nullptr, *d_chunk_search = nullptr, *d_chunk_first = nullptr;
    lxk::PoolSearch* d_searches = nullptr;
    uint32_t* d_head = nullptr;
    uint32_t* d_hit_count = nullptr;
    lxk::PoolHit* d_hits = nullptr;
    uint32_t* d_scalars = nullptr;  // staging for a submission's scalars
    uint32_t* d_lane_map = nullptr;
    uint32_t* h_hit_count = nullptr;  // pinned
    lxk::PoolHit* h_hits = nullptr;   // pinned
    std::vector<int32_t> chunk_owner;  // search slot or -1
    std::vector<uint32_t> h_chunk_search, h_chunk_first;  // mirrors of the device chunk tables
    std::vector<uint32_t> free_chunks;
    std::vector<Search> searches;
    bool queue_dirty = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    uint32_t graph_groups = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;
    fe tu[LXMFV_MAX_HALF_GROUP + 1], tv[LXMFV_MAX_HALF_GROUP + 1];
    std::string err;
};

namespace {

int pfail(lxmfv_pool* p, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (p) p->err = buf;
    return code;
}

#define PCU(p, call)                                                                          \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return pfail((p), LXMFV_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                                 \
    } while (0)

fe words8(const uint32_t w[8]) {
    fe x;
    for (int i = 0; i < 8; i++) x.v[i] = w[i];
    return x;
}

fe pool_u8b() {
    static const uint32_t W[8] = {0x48c99968u, 0xf1716fedu, 0xad74a91eu, 0x7a78edcau,
                                  0xc8b65ca1u, 0xd83b884du, 0xaad65c2du, 0x275fa6d7u};
    return words8(W);
}

fe pool_v8b() {  // the even square root, as in lxmfv.cu
    static const uint32_t W[8] = {0x9f728718u, 0xc5296d6eu, 0x70c591f9u, 0x4f479c67u,
                                  0x4066b08cu, 0x8dcf4469u, 0x8fb939e4u, 0x6085bbbau};
    return words8(W);
}

template <int M>
const void* pool_kernel_ptr() {
    return (const void*)lxk::pool_walk_kernel<M>;
}

const void* pool_kernel_for(uint32_t batch) {
    switch (batch) {
        case 64: return pool_kernel_ptr<32>();
        case 128: return pool_kernel_ptr<64>();
        case 256: return pool_kernel_ptr<128>();
        case 512: return pool_kernel_ptr<256>();
        case 1024: return pool_kernel_ptr<512>();
    }
    return nullptr;
}

template <int M>
void launch_pool(lxmfv_pool* p, uint32_t groups) {
    lxk::PoolArgs<M> a;
    a.state = p->d_state;
    a.ns = p->d_ns;
    a.capacity = p->capacity;
    a.queue = p->d_queue;
    a.n_queue = p->d_nq;
    a.chunk_search = p->d_chunk_search;
    a.chunk_first = p->d_chunk_first;
    a.searches = p->d_searches;
    a.head = p->d_head;
    a.groups = groups;
    a.hit_count = p->d_hit_count;
    a.hits = p->d_hits;
    a.max_hits = p->max_hits;
    a.one = 1;
    if constexpr (M <= 256) {
        for (int i = 0; i <= M; i++) {
            a.t.u[i] = p->tu[i];
            a.t.v[i] = p->tv[i];
        }
    }
    lxk::pool_walk_kernel<M><<<p->sms, 32 * lxk::kPoolWarps, 0, p->stream>>>(a);
}

void launch_pool_any(lxmfv_pool* p, uint32_t groups) {
    switch (p->batch) {
        case 64: launch_pool<32>(p, groups); break;
        case 128: launch_pool<64>(p, groups); break;
        case 256: launch_pool<128>(p, groups); break;
        case 512: launch_pool<256>(p, groups); break;
        default: launch_pool<512>(p, groups); break;
    }
}

int rebuild_queue(lxmfv_pool* p) {
    std::vector<uint32_t> q;
    q.reserve(p->chunks);
    for (const auto& s : p->searches)
        if (s.active) q.insert(q.end(), s.chunks.begin(), s.chunks.end());
    const uint32_t nq = (uint32_t)q.size();
    if (nq) PCU(p, cudaMemcpyAsync(p->d_queue, q.data(), sizeof(uint32_t) * nq, cudaMemcpyHostToDevice, p->stream));
    PCU(p, cudaMemcpyAsync(p->d_chunk_search, p->h_chunk_search.data(), sizeof(uint32_t) * p->chunks,
                           cudaMemcpyHostToDevice, p->stream));
    PCU(p, cudaMemcpyAsync(p->d_chunk_first, p->h_chunk_first.data(), sizeof(uint32_t) * p->chunks,
                           cudaMemcpyHostToDevice, p->stream));
    PCU(p, cudaMemcpyAsync(p->d_nq, &nq, sizeof nq, cudaMemcpyHostToDevice, p->stream));
    // The copies above read host memory that is gone after return: wait for them.
    PCU(p, cudaStreamSynchronize(p->stream));
    p->queue_dirty = false;
    return LXMFV_OK;
}

int capture_step(lxmfv_pool* p, uint32_t groups) {
    if (p->graph_exec) {
        cudaGraphExecDestroy(p->graph_exec);
        p->graph_exec = nullptr;
    }
    if (p->graph) {
        cudaGraphDestroy(p->graph);
        p->graph = nullptr;
    }
    PCU(p, cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(p->d_head, 0, sizeof(uint32_t), p->stream);
    launch_pool_any(p, groups);
    cudaMemcpyAsync(p->h_hit_count, p->d_hit_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, p->stream);
    cudaMemcpyAsync(p->h_hits, p->d_hits, sizeof(lxk::PoolHit) * p->max_hits, cudaMemcpyDeviceToHost, p->stream);
    PCU(p, cudaStreamEndCapture(p->stream, &p->graph));
    PCU(p, cudaGraphInstantiate(&p->graph_exec, p->graph, 0));
    p->graph_groups = groups;
    return LXMFV_OK;
}

}  // namespace

// No exception crosses the C ABI: a host allocation failure (the chunk tables
// and lane maps grow with the capacity, up to 2^28 lanes) becomes
// LXMFV_ERR_NOMEM, with a message when the pool exists (*pp, read after the
// body ran: lxmfv_pool_open hands its pool out before it can fail).
template <class Fn>
static int no_throw(lxmfv_pool* const* pp, Fn&& body) noexcept {
    const char* msg = "unexpected exception";
    int rc = LXMFV_ERR_STATE;
    try {
        return body();
    } catch (const std::bad_alloc&) {
        msg = "out of host memory";
        rc = LXMFV_ERR_NOMEM;
    } catch (...) {
    }
    if (pp && *pp) try { (*pp)->err = msg; } catch (...) {}
    return rc;
}

extern "C" {

static int pool_open_body(const lxmfv_pool_options* opts, lxmfv_pool** out) {
    if (!out) return LXMFV_ERR_ARG;
    *out = nullptr;
    lxmfv_pool* p = new (std::nothrow) lxmfv_pool();
    if (!p) return LXMFV_ERR_NOMEM;
    *out = p;
    lxmfv_pool_options o{};
    if (opts) o = *opts;
    p->device = o.device;
    p->batch = o.batch ? o.batch : 1024;  // 0: the autotuner's choice on the batched mix
    p->m = p->batch / 2;
    if (!pool_kernel_for(p->batch)) return pfail(p, LXMFV_ERR_ARG, "batch %u: the pool walks groups of 64, 128, 256, 512 or 1024", p->batch);
    p->max_searches = o.max_searches ? o.max_searches : 4096;
    p->max_hits = o.max_hits ? o.max_hits : 65536;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return pfail(p, LXMFV_ERR_CUDA, "no CUDA device: %s", e != cudaSuccess ? cudaGetErrorString(e) : "none found");
    if (p->device < 0 || p->device >= count) return pfail(p, LXMFV_ERR_ARG, "device %d out of range", p->device);
    PCU(p, cudaSetDevice(p->device));
    cudaDeviceProp prop;
    PCU(p, cudaGetDeviceProperties(&prop, p->device));
    if (prop.major != 10 || prop.minor != 0)
        return pfail(p, LXMFV_ERR_CUDA, "%s is compute %d.%d; this library is built for sm_100a (B200) only", prop.name,
                     prop.major, prop.minor);
    p->sms = prop.multiProcessorCount;
    int per_sm = 0;
    PCU(p, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pool_kernel_for(p->batch), 32 * lxk::kPoolWarps, 0));
    if (per_sm < 1) return pfail(p, LXMFV_ERR_CUDA, "the pool kernel cannot be resident");
    // Capacity: the memory budget over the bytes a lane needs (state 64, walk
    // index 8, submission staging 36), in whole chunks.
    const uint64_t per_lane = 64 + 8 + 32 + 4;
    uint64_t cap = o.capacity_lanes;
    if (!cap && o.memory_budget) cap = o.memory_budget / per_lane;
    if (!cap) cap = 1u << 20;
    cap = (cap / 32) * 32;
    if (cap == 0 || cap > (1u << 28)) return pfail(p, LXMFV_ERR_ARG, "capacity of %llu lanes is out of range", (unsigned long long)cap);
    p->capacity = (uint32_t)cap;
    p->chunks = p->capacity / 32;
    if (o.stream) {
        p->stream = (cudaStream_t)o.stream;
    } else {
        PCU(p, cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
        p->own_stream = true;
    }
    PCU(p, cudaEventCreate(&p->ev0));
    PCU(p, cudaEventCreate(&p->ev1));
    PCU(p, cudaMalloc(&p->d_state, (size_t)p->capacity * 16 * sizeof(uint32_t)));
    PCU(p, cudaMalloc(&p->d_ns, (size_t)p->capacity * sizeof(uint64_t)));
    PCU(p, cudaMalloc(&p->d_queue, (size_t)p->chunks * sizeof(uint32_t)));
    PCU(p, cudaMalloc(&p->d_nq, sizeof(uint32_t)));
    PCU(p, cudaMalloc(&p->d_chunk_search, (size_t)p->chunks * sizeof(uint32_t)));
    PCU(p, cudaMalloc(&p->d_chunk_first, (size_t)p->chunks * sizeof(uint32_t)));
    PCU(p, cudaMalloc(&p->d_searches, (size_t)p->max_searches * sizeof(lxk::PoolSearch)));
    PCU(p, cudaMalloc(&p->d_head, sizeof(uint32_t)));
    PCU(p, cudaMalloc(&p->d_hit_count, sizeof(uint32_t)));
    PCU(p, cudaMalloc(&p->d_hits, (size_t)p->max_hits * sizeof(lxk::PoolHit)));
    PCU(p, cudaMalloc(&p->d_scalars, (size_t)p->capacity * 32));
    PCU(p, cudaMalloc(&p->d_lane_map, (size_t)p->capacity * sizeof(uint32_t)));
    PCU(p, cudaMallocHost(&p->h_hit_count, sizeof(uint32_t)));
    PCU(p, cudaMallocHost(&p->h_hits, (size_t)p->max_hits * sizeof(lxk::PoolHit)));
    *p->h_hit_count = 0;
    PCU(p, cudaMemsetAsync(p->d_hit_count, 0, sizeof(uint32_t), p->stream));
    PCU(p, cudaMemsetAsync(p->d_nq, 0, sizeof(uint32_t), p->stream));
    PCU(p, cudaMemsetAsync(p->d_chunk_search, 0, (size_t)p->chunks * sizeof(uint32_t), p->stream));
    p->chunk_owner.assign(p->chunks, -1);
    p->h_chunk_search.assign(p->chunks, 0);
    p->h_chunk_first.assign(p->chunks, 0);
    p->free_chunks.resize(p->chunks);
    for (uint32_t c = 0; c < p->chunks; c++) p->free_chunks[c] = p->chunks - 1 - c;  // pop_back gives 0, 1, ...
    p->searches.resize(p->max_searches);
    // The grouped walk's table (as lxmfv_open builds it).
    // Both scratch buffers are freed on every path, including a failed allocation of the second.
    fe *du = nullptr, *dv = nullptr;
    e = cudaMalloc(&du, sizeof(fe) * (p->m + 1));
    if (e == cudaSuccess) e = cudaMalloc(&dv, sizeof(fe) * (p->m + 1));
    if (e == cudaSuccess) {
        lxk::group_table_kernel<<<1, ((p->m + 1 + 31) / 32) * 32, 0, p->stream>>>(du, dv, p->m, pool_u8b(),
                                                                                  pool_v8b());
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->tu, du, sizeof(fe) * (p->m + 1), cudaMemcpyDeviceToHost, p->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->tv, dv, sizeof(fe) * (p->m + 1), cudaMemcpyDeviceToHost, p->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    cudaFree(du);
    cudaFree(dv);
    if (e == cudaSuccess && p->m > 256) {
        // Groups of 1024: the table goes to this module's constant memory (the
        // same bytes for every pool on the device).
        e = cudaMemcpyToSymbolAsync(lxk::c_group_u, p->tu, sizeof(fe) * (p->m + 1), 0, cudaMemcpyHostToDevice,
                                    p->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyToSymbolAsync(lxk::c_group_v, p->tv, sizeof(fe) * (p->m + 1), 0, cudaMemcpyHostToDevice,
                                        p->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    }
    if (e != cudaSuccess) return pfail(p, LXMFV_ERR_CUDA, "pool table: %s", cudaGetErrorString(e));
    p->err.clear();
    return LXMFV_OK;
}

const char* lxmfv_pool_last_error(const lxmfv_pool* p) { return p ? p->err.c_str() : "null pool"; }

int lxmfv_pool_info(const lxmfv_pool* p, lxmfv_pool_info_t* info) {
    if (!p || !info) return LXMFV_ERR_ARG;
    memset(info, 0, sizeof *info);
    info->capacity_lanes = p->capacity;
    info->free_lanes = (uint32_t)p->free_chunks.size() * 32;
    for (const auto& s : p->searches)
        if (s.active) {
            info->active_searches++;
            info->active_lanes += s.lanes;
        }
    info->batch = p->batch;
    info->sms = (uint32_t)p->sms;
    return LXMFV_OK;
}

static int pool_submit_body(lxmfv_pool* p, const lxmfv_search_desc* d, const uint8_t* scalars, uint32_t* search_id) {
    if (!p || !d || !scalars || !search_id) return pfail(p, LXMFV_ERR_ARG, "null argument");
    if (d->lanes == 0 || d->lanes % 32) return pfail(p, LXMFV_ERR_ARG, "lanes %u: a positive multiple of 32", d->lanes);
    const uint32_t need = d->lanes / 32;
    if (need > p->free_chunks.size())
        return pfail(p, LXMFV_ERR_OVERFLOW, "%u lanes asked, %zu free", d->lanes, p->free_chunks.size() * 32);
    uint32_t slot = 0;
    while (slot < p->max_searches && p->searches[slot].active) slot++;
    if (slot == p->max_searches) return pfail(p, LXMFV_ERR_OVERFLOW, "all %u search slots are in use", p->max_searches);
    for (uint32_t t = 0; t < d->lanes; t++) {
        const uint8_t* k = scalars + 32 * (size_t)t;
        if ((k[0] & 7) != 0 || (k[31] & 0xC0) != 0x40)
            return pfail(p, LXMFV_ERR_ARG, "scalar %u is not clamped", t);
    }
    PCU(p, cudaSetDevice(p->device));
    auto& s = p->searches[slot];
    s.chunks.clear();
    for (uint32_t i = 0; i < need; i++) {
        s.chunks.push_back(p->free_chunks.back());
        p->free_chunks.pop_back();
    }
    std::sort(s.chunks.begin(), s.chunks.end());
    std::vector<uint32_t> lane_map(d->lanes);
    for (uint32_t i = 0; i < need; i++) {
        const uint32_t c = s.chunks[i];
        p->chunk_owner[c] = (int32_t)slot;
        p->h_chunk_search[c] = slot;
        p->h_chunk_first[c] = 32 * i;
        for (uint32_t j = 0; j < 32; j++) lane_map[32 * i + j] = 32 * c + j;
    }
    lxk::PoolSearch ps;
    memset(&ps, 0, sizeof ps);
    ps.ac.one = 1;
    memcpy(ps.ac.ed, d->ed, sizeof ps.ac.ed);
    memcpy(ps.ac.nh, d->name_hash, sizeof ps.ac.nh);
    memcpy(ps.ac.want, d->want, sizeof ps.ac.want);
    memcpy(ps.ac.mask, d->mask, sizeof ps.ac.mask);
    cudaError_t e = cudaMemcpyAsync(&p->d_searches[slot], &ps, sizeof ps, cudaMemcpyHostToDevice, p->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->d_scalars, scalars, (size_t)d->lanes * 32, cudaMemcpyHostToDevice, p->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_lane_map, lane_map.data(), sizeof(uint32_t) * d->lanes, cudaMemcpyHostToDevice, p->stream);
    if (e == cudaSuccess) {
        lxk::pool_start_kernel<<<(d->lanes + 127) / 128, 128, 0, p->stream>>>(
            p->d_state, p->d_ns, p->capacity, p->d_scalars, p->d_lane_map, d->lanes, p->m, pool_u8b(), pool_v8b());
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) {
        for (uint32_t c : s.chunks) {
            p->chunk_owner[c] = -1;
            p->free_chunks.push_back(c);
        }
        s.chunks.clear();
        return pfail(p, LXMFV_ERR_CUDA, "submit: %s", cudaGetErrorString(e));
    }
    s.active = true;
    s.lanes = d->lanes;
    s.keys_per_lane = 0;
    p->queue_dirty = true;
    *search_id = slot;
    p->err.clear();
    return LXMFV_OK;
}

// Admission of many searches with one start kernel and no host wait.  The
// staging buffers (d_scalars, d_lane_map) are rewritten only by later copies on
// the same stream, so they are never overwritten before this kernel has read
// them, and every host source is copied out before its cudaMemcpyAsync
// returns (pageable memory).
static int pool_submit_many_body(lxmfv_pool* p, const lxmfv_search_desc* descs, uint32_t n, const uint8_t* scalars,
                                 uint32_t* search_ids, uint32_t* n_admitted) {
    if (!p || !n_admitted || (n && (!descs || !scalars || !search_ids))) return pfail(p, LXMFV_ERR_ARG, "null argument");
    *n_admitted = 0;
    if (n == 0) return LXMFV_OK;
    // How many fit, in order; every admitted search's descriptor and scalars are checked first.
    uint64_t free_lanes = (uint64_t)p->free_chunks.size() * 32, lanes_total = 0;
    uint32_t free_slots = 0;
    for (const auto& s : p->searches) free_slots += s.active ? 0 : 1;
    uint32_t take = 0;
    size_t off = 0;
    for (; take < n; take++) {
        const lxmfv_search_desc& d = descs[take];
        if (d.lanes == 0 || d.lanes % 32)
            return pfail(p, LXMFV_ERR_ARG, "search %u: lanes %u, a positive multiple of 32", take, d.lanes);
        if (lanes_total + d.lanes > free_lanes || take >= free_slots) break;
        for (uint32_t t = 0; t < d.lanes; t++) {
            const uint8_t* k = scalars + off + 32 * (size_t)t;
            if ((k[0] & 7) != 0 || (k[31] & 0xC0) != 0x40)
                return pfail(p, LXMFV_ERR_ARG, "search %u: scalar %u is not clamped", take, t);
        }
        lanes_total += d.lanes;
        off += 32 * (size_t)d.lanes;
    }
    if (take == 0)
        return pfail(p, LXMFV_ERR_OVERFLOW, "%u lanes asked, %llu free, %u slots free", descs[0].lanes,
                     (unsigned long long)free_lanes, free_slots);
    PCU(p, cudaSetDevice(p->device));
    std::vector<uint32_t> lane_map(lanes_total);
    std::vector<uint32_t> slots(take);
    uint32_t slot = 0;
    size_t at = 0;
    cudaError_t e = cudaSuccess;
    uint32_t done = 0;
    for (; done < take; done++) {
        const lxmfv_search_desc& d = descs[done];
        while (p->searches[slot].active) slot++;  // a free slot exists: counted above
        auto& s = p->searches[slot];
        s.chunks.clear();
        for (uint32_t i = 0; i < d.lanes / 32; i++) {
            s.chunks.push_back(p->free_chunks.back());
            p->free_chunks.pop_back();
        }
        std::sort(s.chunks.begin(), s.chunks.end());
        for (uint32_t i = 0; i < d.lanes / 32; i++) {
            const uint32_t c = s.chunks[i];
            p->chunk_owner[c] = (int32_t)slot;
            p->h_chunk_search[c] = slot;
            p->h_chunk_first[c] = 32 * i;
            for (uint32_t j = 0; j < 32; j++) lane_map[at + 32 * i + j] = 32 * c + j;
        }
        at += d.lanes;
        s.active = true;  // claimed, so the next search takes another slot
        s.lanes = d.lanes;
        s.keys_per_lane = 0;
        slots[done] = slot;
        lxk::PoolSearch ps;
        memset(&ps, 0, sizeof ps);
        ps.ac.one = 1;
        memcpy(ps.ac.ed, d.ed, sizeof ps.ac.ed);
        memcpy(ps.ac.nh, d.name_hash, sizeof ps.ac.nh);
        memcpy(ps.ac.want, d.want, sizeof ps.ac.want);
        memcpy(ps.ac.mask, d.mask, sizeof ps.ac.mask);
        e = cudaMemcpyAsync(&p->d_searches[slot], &ps, sizeof ps, cudaMemcpyHostToDevice, p->stream);
        if (e != cudaSuccess) {
            done++;
            break;
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->d_scalars, scalars, 32 * (size_t)lanes_total, cudaMemcpyHostToDevice, p->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_lane_map, lane_map.data(), sizeof(uint32_t) * lanes_total, cudaMemcpyHostToDevice,
                            p->stream);
    if (e == cudaSuccess) {
        lxk::pool_start_kernel<<<(unsigned)((lanes_total + 127) / 128), 128, 0, p->stream>>>(
            p->d_state, p->d_ns, p->capacity, p->d_scalars, p->d_lane_map, (uint32_t)lanes_total, p->m, pool_u8b(),
            pool_v8b());
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        for (uint32_t i = 0; i < done; i++) {
            auto& s = p->searches[slots[i]];
            for (uint32_t c : s.chunks) {
                p->chunk_owner[c] = -1;
                p->free_chunks.push_back(c);
            }
            s.chunks.clear();
            s.active = false;
            s.lanes = 0;
        }
        return pfail(p, LXMFV_ERR_CUDA, "submit: %s", cudaGetErrorString(e));
    }
    for (uint32_t i = 0; i < take; i++) search_ids[i] = slots[i];
    *n_admitted = take;
    p->queue_dirty = true;
    p->err.clear();
    return LXMFV_OK;
}

static int pool_retire_body(lxmfv_pool* p, uint32_t search_id) {
    if (!p) return LXMFV_ERR_ARG;
    if (search_id >= p->max_searches || !p->searches[search_id].active)
        return pfail(p, LXMFV_ERR_ARG, "search %u is not active", search_id);
    auto& s = p->searches[search_id];
    for (uint32_t c : s.chunks) {
        p->chunk_owner[c] = -1;
        p->free_chunks.push_back(c);
    }
    s.chunks.clear();
    s.active = false;
    s.lanes = 0;
    p->queue_dirty = true;
    p->err.clear();
    return LXMFV_OK;
}

static int pool_step_body(lxmfv_pool* p, uint32_t groups) {
    if (!p) return LXMFV_ERR_ARG;
    if (groups == 0 || groups > (1u << 16)) return pfail(p, LXMFV_ERR_ARG, "groups %u: 1 .. 65536", groups);
    PCU(p, cudaSetDevice(p->device));
    if (p->queue_dirty)
        if (int rc = rebuild_queue(p)) return rc;
    if (!p->graph_exec || p->graph_groups != groups)
        if (int rc = capture_step(p, groups)) return rc;
    PCU(p, cudaEventRecord(p->ev0, p->stream));
    PCU(p, cudaGraphLaunch(p->graph_exec, p->stream));
    PCU(p, cudaEventRecord(p->ev1, p->stream));
    p->timed = true;
    for (auto& s : p->searches)
        if (s.active) s.keys_per_lane += (uint64_t)groups * p->batch;
    return LXMFV_OK;
}

int lxmfv_pool_poll(lxmfv_pool* p, lxmfv_pool_hit* hits, uint32_t cap, uint32_t* n_hits) {
    if (!p || !n_hits) return pfail(p, LXMFV_ERR_ARG, "null argument");
    PCU(p, cudaSetDevice(p->device));
    PCU(p, cudaStreamSynchronize(p->stream));
    // The last step's graph copied the hit queue to pinned memory.
    const uint32_t count = *p->h_hit_count;
    const uint32_t stored = std::min(count, p->max_hits);
    const uint32_t give = hits ? std::min(stored, cap) : 0;
    for (uint32_t i = 0; i < give; i++) {
        hits[i].search = p->h_hits[i].search;
        hits[i].lane = p->h_hits[i].lane;
        hits[i].n = p->h_hits[i].n;
    }
    *n_hits = count;
    PCU(p, cudaMemsetAsync(p->d_hit_count, 0, sizeof(uint32_t), p->stream));
    PCU(p, cudaStreamSynchronize(p->stream));
    *p->h_hit_count = 0;
    p->err.clear();
    return LXMFV_OK;
}

uint64_t lxmfv_pool_keys_per_lane(const lxmfv_pool* p, uint32_t search_id) {
    if (!p || search_id >= p->max_searches) return 0;
    return p->searches[search_id].keys_per_lane;
}

float lxmfv_pool_last_step_ms(const lxmfv_pool* p) {
    if (!p || !p->timed) return -1.0f;
    float ms = -1.0f;
    if (cudaEventSynchronize(p->ev1) != cudaSuccess) return -1.0f;
    if (cudaEventElapsedTime(&ms, p->ev0, p->ev1) != cudaSuccess) return -1.0f;
    return ms;
}

int lxmfv_pool_open(const lxmfv_pool_options* opts, lxmfv_pool** out) {
    return no_throw(out, [&] { return pool_open_body(opts, out); });
}

int lxmfv_pool_submit(lxmfv_pool* p, const lxmfv_search_desc* d, const uint8_t* scalars, uint32_t* search_id) {
    return no_throw(&p, [&] { return pool_submit_body(p, d, scalars, search_id); });
}

int lxmfv_pool_submit_many(lxmfv_pool* p, const lxmfv_search_desc* descs, uint32_t n, const uint8_t* scalars,
                           uint32_t* search_ids, uint32_t* n_admitted) {
    return no_throw(&p, [&] { return pool_submit_many_body(p, descs, n, scalars, search_ids, n_admitted); });
}

int lxmfv_pool_retire(lxmfv_pool* p, uint32_t search_id) {
    return no_throw(&p, [&] { return pool_retire_body(p, search_id); });
}

int lxmfv_pool_step(lxmfv_pool* p, uint32_t groups) {
    return no_throw(&p, [&] { return pool_step_body(p, groups); });
}

void lxmfv_pool_close(lxmfv_pool* p) {
    if (!p) return;
    if (p->sms) {
        cudaSetDevice(p->device);
        if (p->stream) cudaStreamSynchronize(p->stream);
        if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
        if (p->graph) cudaGraphDestroy(p->graph);
        cudaFree(p->d_state);
        cudaFree(p->d_ns);
        cudaFree(p->d_queue);
        cudaFree(p->d_nq);
        cudaFree(p->d_chunk_search);
        cudaFree(p->d_chunk_first);
        cudaFree(p->d_searches);
        cudaFree(p->d_head);
        cudaFree(p->d_hit_count);
        cudaFree(p->d_hits);
        cudaFree(p->d_scalars);
        cudaFree(p->d_lane_map);
        cudaFreeHost(p->h_hit_count);
        cudaFreeHost(p->h_hits);
        if (p->ev0) cudaEventDestroy(p->ev0);
        if (p->ev1) cudaEventDestroy(p->ev1);
        if (p->own_stream && p->stream) cudaStreamDestroy(p->stream);
    }
    delete p;
}

}  // extern "C"
