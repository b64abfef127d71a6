// Batch inversion for callers that cannot allocate device memory.
//
// Some callers of this library are not allowed to call cudaMalloc or
// cudaFree: a host runtime that owns every device allocation itself (an
// engine with its own memory pool, a plugin that is handed device buffers and
// must not grow the process's footprint behind the host's back), or a
// latency-critical loop where cudaFree's implicit device synchronisation is
// not acceptable.  lxmfv_fe_op allocates its staging and working buffers on
// every call, so it is closed to them.
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
//     aligned, `count` elements of 8 little-endian words each; d_out may be
//     d_a (in place), but the two ranges may not otherwise overlap;
//   - count <= LXMFV_STATIC_SCRATCH_ELEMS, else LXMFV_ERR_ARG and nothing runs;
//   - the first call in a CUDA context (the device's primary context, made
//     current by the runtime) looks up the scratch array's device address
//     with cudaGetSymbolAddress.  After cudaDeviceReset the runtime gives
//     the device a new context, and the next call looks the address up
//     again;
//   - every call shares the one array: calls whose kernels overlap on the
//     GPU (two streams, or two host threads) race on it and must be ordered
//     by the caller.  Nothing in the array needs to start at zero: each
//     prefix product is written before it is read.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/lxmfv.h"
#include "fe25519.cuh"

namespace {

// The scratch: prefix products of the elements of one call.
static __device__ __align__(256) fe g_static_scratch[LXMFV_STATIC_SCRATCH_ELEMS];

// The scratch's device address per device, with the id of the context it was
// looked up in (a context id is unique for the life of the process).
constexpr int kMaxDevices = 64;
struct ScratchAddr {
    unsigned long long ctx_id;
    fe* addr;
};
ScratchAddr g_scratch[kMaxDevices];
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
// `out`.  `out` may be `a`: each element is read before its inverse is
// stored, and a thread touches only its own group.
__global__ void fe_batch_invert_scratch_kernel(const uint32_t* a, uint32_t* out, uint64_t count, uint32_t group,
                                               fe* __restrict__ scratch) {
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
            const fe ai = load8_drop255(a + 8 * (base + i));
            store8(out + 8 * (base + i), fe_canon(fe_mul(inv, scratch[base + i])));
            inv = fe_mul(inv, ai);
        }
    }
}

int say(char* err, size_t err_len, int code, const char* msg) {
    if (err && err_len) snprintf(err, err_len, "%s", msg);
    return code;
}

// The id of the calling thread's current context, or 0 when none is current
// (or the driver cannot say).  The functions come from the driver through
// the runtime, so the library needs no link against libcuda.
unsigned long long current_ctx_id() {
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 4000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f);
    });
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
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
    {
        // In place (d_out == d_a) is fine; any other overlap would let one
        // thread's stores reach the elements another thread still reads.
        const uintptr_t a0 = (uintptr_t)d_a, o0 = (uintptr_t)d_out, bytes = (uintptr_t)count * 32u;
        if (a0 != o0 && a0 < o0 + bytes && o0 < a0 + bytes)
            return say(err, err_len, LXMFV_ERR_ARG, "input and output overlap without being the same buffer");
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return say(err, err_len, LXMFV_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return say(err, err_len, LXMFV_ERR_STATE, "device ordinal out of range");
    fe* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        const unsigned long long id = current_ctx_id();
        if (id != 0 && g_scratch[dev].addr && g_scratch[dev].ctx_id == id) {
            scratch = g_scratch[dev].addr;
        } else {
            // Set-up for this device's context, with the device current: the
            // array's name in host code is only a host-side stand-in, never a
            // device address, so its device address is looked up here.  This
            // also makes the runtime's context current on this thread.
            e = cudaGetSymbolAddress((void**)&scratch, g_static_scratch);
            if (e != cudaSuccess || !scratch)
                return say(err, err_len, LXMFV_ERR_CUDA,
                           e != cudaSuccess ? cudaGetErrorString(e) : "no address for the scratch array");
            g_scratch[dev].ctx_id = current_ctx_id();
            g_scratch[dev].addr = scratch;
        }
    }
    const unsigned groups = (unsigned)((count + group - 1) / group);
    const unsigned blocks = (groups + 127) / 128;
    fe_batch_invert_scratch_kernel<<<blocks, 128, 0, (cudaStream_t)stream>>>(d_a, d_out, count, group, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return say(err, err_len, LXMFV_ERR_CUDA, cudaGetErrorString(e));
    return LXMFV_OK;
}
