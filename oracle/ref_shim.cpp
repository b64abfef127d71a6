// Host build of the reference's own GPU kernel body, for use as a checker.
//
// TEST INFRASTRUCTURE ONLY.  This file contains no reference code: it
// supplies the portability macros that src/gpu/kernel.cu:4-17 supplies for
// CUDA (here: plain C++ on the CPU) and then includes the reference's
// src/gpu/common.h from where it lies, read-only (the include path is given
// by oracle/Makefile).  The result, oracle/_ref/libref.so, is never shipped
// and never committed; it runs the reference's exact arithmetic on the CPU:
//   - init_thread / walk_thread            common.h:261-365
//   - fe_mul / fe_sq / fe_invert           common.h:75-128
//   - fe_from_words / fe_to_words          common.h:131-174
//   - lxmf_address (three compressions)    common.h:221-253
#include <cstdint>
#include <cstring>
#include <pthread.h>
#include <ctime>

typedef int32_t i32;
typedef uint32_t u32;
typedef int64_t i64;
typedef uint64_t u64;

#define FN static inline
#define TABLE static const
#define GLOBAL
#define LOCAL_U32_PTR u32*
#define LOCAL_I64_PTR i64*
#define HIT_COUNTER u32
#define ATOMIC_INC(p) __atomic_fetch_add((p), 1u, __ATOMIC_RELAXED)
static inline u32 ref_rotr(u32 x, int n) { return (x >> n) | (x << (32 - n)); }
#define rotr(x, n) ref_rotr((x), (n))
#define bswap(x) __builtin_bswap32(x)
#ifndef BATCH
#define BATCH 64
#endif

#include "common.h"

extern "C" {

int ref_batch(void) { return BATCH; }

void ref_init_walk(i32* state, const u32* u_prev_cur, u32 threads) {
    for (u32 t = 0; t < threads; t++) init_thread(t, state, u_prev_cur);
}

void ref_walk(i32* state, u64* ns, u32 threads, u32 iters, const u32* ed, u32 nh0, u32 nh1, u32 nh2,
              const u32* want, const u32* mask, u32* hit_count, u64* hits, u32 max_hits, u32* dump,
              u32 dump_threads, const u32* q_words) {
    for (u32 t = 0; t < threads; t++)
        walk_thread(t, state, ns, iters, ed, nh0, nh1, nh2, want, mask, hit_count, hits, max_hits, dump,
                    dump_threads, q_words);
}

void ref_lxmf_address(const u32* u, const u32* ed, const u32* nh, u32* out, u64 count) {
    for (u64 i = 0; i < count; i++) {
        u32 ul[8], el[8], nl[3], o[4];
        for (int k = 0; k < 8; k++) { ul[k] = u[8 * i + k]; el[k] = ed[8 * i + k]; }
        for (int k = 0; k < 3; k++) nl[k] = nh[k];
        lxmf_address(ul, el, nl, o);
        for (int k = 0; k < 4; k++) out[4 * i + k] = o[k];
    }
}

// op: 0 mul, 1 square, 2 invert; inputs through fe_from_words (bit 255
// dropped), outputs through fe_to_words (canonical).
void ref_fe_op(int op, const u32* a, const u32* b, u32* out, u64 count) {
    for (u64 i = 0; i < count; i++) {
        u32 w[8];
        for (int k = 0; k < 8; k++) w[k] = a[8 * i + k];
        fe x = fe_from_words(w), r;
        if (op == 0) {
            for (int k = 0; k < 8; k++) w[k] = b[8 * i + k];
            r = fe_mul(x, fe_from_words(w));
        } else if (op == 1) {
            r = fe_sq(x);
        } else {
            r = fe_invert(x);
        }
        fe_to_words(r, out + 8 * i);
    }
}

// Montgomery's trick over groups of `group` (<= 256) elements, with the
// walk's structure (common.h:326-356).
void ref_fe_batch_invert(const u32* a, u32* out, u64 count, int group) {
    static thread_local fe zs[256], prefix[256];
    for (u64 g0 = 0; g0 < count; g0 += (u64)group) {
        int len = (int)((count - g0) < (u64)group ? (count - g0) : (u64)group);
        fe acc = fe_one();
        for (int i = 0; i < len; i++) {
            u32 w[8];
            for (int k = 0; k < 8; k++) w[k] = a[8 * (g0 + i) + k];
            zs[i] = fe_from_words(w);
            prefix[i] = acc;
            acc = fe_mul(acc, zs[i]);
        }
        fe inv = fe_invert(acc);
        for (int i = len - 1; i >= 0; i--) {
            fe_to_words(fe_mul(inv, prefix[i]), out + 8 * (g0 + i));
            inv = fe_mul(inv, zs[i]);
        }
    }
}

// Timed CPU run of walk_thread: `workers` POSIX threads share `threads`
// walker lanes (set up by ref_init_walk from u_prev_cur) and each lane walks
// `iters` batches.  Returns keys per second (wall clock).
struct ref_job {
    u32 lo, hi, iters;
    i32* state; u64* ns;
    const u32 *ed, *want, *mask, *q;
    u32 nh0, nh1, nh2;
    u32* hit_count; u64* hits; u32 max_hits;
};

static void* ref_job_run(void* arg) {
    ref_job* j = (ref_job*)arg;
    for (u32 t = j->lo; t < j->hi; t++)
        walk_thread(t, j->state, j->ns, j->iters, j->ed, j->nh0, j->nh1, j->nh2, j->want, j->mask, j->hit_count,
                    j->hits, j->max_hits, nullptr, 0, j->q);
    return nullptr;
}

double ref_bench_walk(int workers, i32* state, u64* ns, u32 threads, u32 iters, const u32* ed, u32 nh0, u32 nh1,
                      u32 nh2, const u32* want, const u32* mask, u32* hit_count, u64* hits, u32 max_hits,
                      const u32* q_words) {
    if (workers < 1) workers = 1;
    ref_job jobs[512];
    pthread_t tid[512];
    if (workers > 512) workers = 512;
    u32 per = (threads + (u32)workers - 1) / (u32)workers;
    int used = 0;
    for (int w = 0; w < workers; w++) {
        u32 lo = (u32)w * per, hi = lo + per > threads ? threads : lo + per;
        if (lo >= hi) break;
        jobs[used] = ref_job{lo, hi, iters, state, ns, ed, want, mask, q_words, nh0, nh1, nh2, hit_count, hits, max_hits};
        used++;
    }
    timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (int w = 0; w < used; w++) pthread_create(&tid[w], nullptr, ref_job_run, &jobs[w]);
    for (int w = 0; w < used; w++) pthread_join(tid[w], nullptr);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    double secs = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    return secs > 0 ? (double)threads * iters * BATCH / secs : 0.0;
}

}  // extern "C"
