// Batch inversion for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: code that runs while a CUDA
// graph is being captured, code inside a host runtime that owns every device
// allocation itself (an embedding engine with its own pool, a plugin that is
// handed device buffers), or code on a path where an allocation's implicit
// device synchronisation is not acceptable.  lxmfv_fe_op allocates its
// staging and working buffers on every call, so it is closed to them.
//
// lxmfv_fe_batch_invert_static does the same batch inversion (Montgomery's
// trick over groups of `group` elements, as lxmfv_fe_op op 3) on buffers the
// caller already owns, and allocates nothing: the kernel's working storage,
// the running prefix products, lives in one file-scope __device__ array of
// LXMFV_STATIC_SCRATCH_ELEMS field elements (4 MiB), which every GPU that
// loads this library holds until the process exits.
//
// Contract (also in include/lxmfv.h):
//   - inputs and outputs are device pointers on the current device, 16-byte
//     aligned, `count` elements of 8 little-endian words each;
//   - count <= LXMFV_STATIC_SCRATCH_ELEMS, else LXMFV_ERR_ARG and nothing runs;
//   - the first call on a device looks up the scratch array's device address
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before any stream capture;
//   - every call shares the one array: calls whose kernels overlap on the
//     GPU (two streams, or two host threads) race on it and must be ordered
//     by the caller.  Nothing in the array needs to start at zero: each
//     prefix product is written before it is read.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/lxmfv.h"
#include "fe25519.cuh"

namespace {

// The scratch: prefix products of the elements of one call.
static __device__ __align__(256) fe g_static_scratch[LXMFV_STATIC_SCRATCH_ELEMS];

constexpr int kMaxDevices = 64;
std::atomic<fe*> g_scratch_addr[kMaxDevices];
std::mutex g_setup_mutex;

__device__ __forceinline__ fe load8_drop255(const uint32_t* p) {
    const uint4* p4 = reinterpret_cast<const uint4*>(p);
    const uint4 lo = p4[0], hi = p4[1];
    fe r;
    r.v[0] = lo.x; r.v[1] = lo.y; r.v[2] = lo.z; r.v[3] = lo.w;
    r.v[4] = hi.x; r.v[5] = hi.y; r.v[6] = hi.z; r.v[7] = hi.w & 0x7fffffffu;
    return r;
}

__device__ __forceinline__ void store8(uint32_t* p, const fe& x) {
    uint4* p4 = reinterpret_cast<uint4*>(p);
    p4[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
    p4[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

// One group per thread: prefix products go to `scratch`, the inverses to
// `out`, which is only written.
__global__ void fe_batch_invert_scratch_kernel(const uint32_t* __restrict__ a, uint32_t* __restrict__ out,
                                               uint64_t count, uint32_t group, fe* __restrict__ scratch) {
    const uint64_t groups = (count + group - 1) / group;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < groups; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = g * group;
        const uint32_t len = (uint32_t)((count - base) < group ? (count - base) : group);
        fe acc = fe_one();
        for (uint32_t i = 0; i < len; i++) {
            scratch[base + i] = acc;
            acc = fe_mul(acc, load8_drop255(a + 8 * (base + i)));
        }
        fe inv = fe_invert(acc);
        for (int i = (int)len - 1; i >= 0; i--) {
            store8(out + 8 * (base + i), fe_canon(fe_mul(inv, scratch[base + i])));
            inv = fe_mul(inv, load8_drop255(a + 8 * (base + i)));
        }
    }
}

int say(char* err, size_t err_len, int code, const char* msg) {
    if (err && err_len) snprintf(err, err_len, "%s", msg);
    return code;
}

}  // namespace

extern "C" int lxmfv_fe_batch_invert_static(const uint32_t* d_a, uint32_t* d_out, uint64_t count, uint32_t group,
                                            void* stream, char* err, size_t err_len) {
    if (err && err_len) err[0] = 0;
    if (!d_a || !d_out) return say(err, err_len, LXMFV_ERR_ARG, "null device pointer");
    if (group < 1 || group > 256) return say(err, err_len, LXMFV_ERR_ARG, "group must be 1..256");
    if (count > LXMFV_STATIC_SCRATCH_ELEMS) {
        char msg[160];
        snprintf(msg, sizeof msg, "count %llu exceeds the static scratch of %u elements",
                 (unsigned long long)count, (unsigned)LXMFV_STATIC_SCRATCH_ELEMS);
        return say(err, err_len, LXMFV_ERR_ARG, msg);
    }
    if ((((uintptr_t)d_a) | ((uintptr_t)d_out)) & 15u)
        return say(err, err_len, LXMFV_ERR_ARG, "device pointers must be 16-byte aligned");
    if (count == 0) return LXMFV_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return say(err, err_len, LXMFV_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return say(err, err_len, LXMFV_ERR_STATE, "device ordinal out of range");
    fe* scratch = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!scratch) {
        // First call on this device (the current one): look up the array's
        // device address.  The array's name in host code is only a host-side
        // stand-in, never a device address.
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        scratch = g_scratch_addr[dev].load(std::memory_order_acquire);
        if (!scratch) {
            e = cudaGetSymbolAddress((void**)&scratch, g_static_scratch);
            if (e != cudaSuccess || !scratch)
                return say(err, err_len, LXMFV_ERR_CUDA,
                           e != cudaSuccess ? cudaGetErrorString(e) : "no address for the scratch array");
            g_scratch_addr[dev].store(scratch, std::memory_order_release);
        }
    }
    const unsigned groups = (unsigned)((count + group - 1) / group);
    const unsigned blocks = (groups + 127) / 128;
    fe_batch_invert_scratch_kernel<<<blocks, 128, 0, (cudaStream_t)stream>>>(d_a, d_out, count, group, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return say(err, err_len, LXMFV_ERR_CUDA, cudaGetErrorString(e));
    return LXMFV_OK;
}
