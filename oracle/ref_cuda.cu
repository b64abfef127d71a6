// Host driver for the reference's own CUDA kernels, for comparison on the
// same GPU.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY: never shipped, never committed as a
// build.  It contains no reference code: it includes the reference's
// src/gpu/kernel.cu (which includes common.h) from where it lies, read-only
// (include path given by oracle/Makefile), compiled ahead of time for sm_100a
// instead of by NVRTC at start-up, and drives init_walk / walk the way the
// reference's CUDA backend does (src/gpu/cuda.rs:33-132): BATCH 64, blocks of
// 128 threads, SMs x 2048 threads by default.
#define BATCH 64
#include "kernel.cu"

#include <cstdio>

extern "C" {

// Runs `steps` launches of the reference's walk (after `warmup` launches) of
// `iters` batches for `threads` lanes set from u_prev_cur (16 LE words per
// lane).  Reports the mean device time per launch and keys/s; the hits of the
// first launch (thread, n pairs, up to 4096) and, when dump is not null, the
// first-batch public keys of the first dump_threads lanes.  Returns 0 or a
// CUDA error code.
int refcu_walk(const u32* u_prev_cur, u32 threads, u32 iters, int warmup, int steps, const u32* ed, u32 nh0, u32 nh1,
               u32 nh2, const u32* want, const u32* mask, const u32* q, double* keys_per_s, float* ms_per_launch,
               u32* n_hits, u64* hits, u32 dump_threads, u32* dump) {
    i32* state = nullptr;
    u64* ns = nullptr;
    u32 *upc = nullptr, *ded = nullptr, *dwant = nullptr, *dmask = nullptr, *dq = nullptr, *dhc = nullptr,
        *ddump = nullptr;
    u64* dhits = nullptr;
    cudaEvent_t e0, e1;
    cudaError_t e = cudaSuccess;
#define T(x) if (e == cudaSuccess) e = (x)
    T(cudaMalloc(&state, (size_t)threads * 40 * 4));
    T(cudaMalloc(&ns, (size_t)threads * 8));
    T(cudaMemset(ns, 0, (size_t)threads * 8));
    T(cudaMalloc(&upc, (size_t)threads * 64));
    T(cudaMemcpy(upc, u_prev_cur, (size_t)threads * 64, cudaMemcpyHostToDevice));
    T(cudaMalloc(&ded, 32));
    T(cudaMalloc(&dwant, 16));
    T(cudaMalloc(&dmask, 16));
    T(cudaMalloc(&dq, 32));
    T(cudaMalloc(&dhc, 4));
    T(cudaMalloc(&dhits, 4096 * 16));
    T(cudaMalloc(&ddump, (size_t)(dump_threads ? dump_threads : 1) * BATCH * 32));
    T(cudaMemcpy(ded, ed, 32, cudaMemcpyHostToDevice));
    T(cudaMemcpy(dwant, want, 16, cudaMemcpyHostToDevice));
    T(cudaMemcpy(dmask, mask, 16, cudaMemcpyHostToDevice));
    T(cudaMemcpy(dq, q, 32, cudaMemcpyHostToDevice));
    T(cudaMemset(dhc, 0, 4));
    T(cudaEventCreate(&e0));
    T(cudaEventCreate(&e1));
    const u32 grid = (threads + 127) / 128;
    if (e == cudaSuccess) {
        init_walk<<<grid, 128>>>(state, upc, threads);
        e = cudaGetLastError();
    }
    float total = 0;
    for (int s = 0; s < warmup + steps && e == cudaSuccess; s++) {
        const u32 dt = (s == 0) ? dump_threads : 0;
        T(cudaEventRecord(e0));
        if (e == cudaSuccess) {
            walk<<<grid, 128>>>(state, ns, threads, iters, ded, nh0, nh1, nh2, dwant, dmask, dhc, dhits, 4096, ddump, dt,
                                dq);
            e = cudaGetLastError();
        }
        T(cudaEventRecord(e1));
        T(cudaEventSynchronize(e1));
        float ms = 0;
        T(cudaEventElapsedTime(&ms, e0, e1));
        if (s == 0) {
            T(cudaMemcpy(n_hits, dhc, 4, cudaMemcpyDeviceToHost));
            T(cudaMemcpy(hits, dhits, 4096 * 16, cudaMemcpyDeviceToHost));
            if (dump && dump_threads)
                T(cudaMemcpy(dump, ddump, (size_t)dump_threads * BATCH * 32, cudaMemcpyDeviceToHost));
        }
        if (s >= warmup) total += ms;
    }
    if (e == cudaSuccess && steps > 0) {
        *ms_per_launch = total / steps;
        *keys_per_s = (double)threads * iters * BATCH / (total / steps * 1e-3);
    }
    cudaFree(state); cudaFree(ns); cudaFree(upc); cudaFree(ded); cudaFree(dwant); cudaFree(dmask); cudaFree(dq);
    cudaFree(dhc); cudaFree(dhits); cudaFree(ddump);
#undef T
    return (int)e;
}

int refcu_default_threads(void) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    return sms * 2048;  // THREADS_PER_SM (cuda.rs:16)
}

}  // extern "C"
