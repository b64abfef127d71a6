/*
 * liblxmfv: the B200-native (sm_100a) key-walk search of lxmf-vanity behind a
 * plain C ABI.
 *
 * The reference (alaistair76/lxmf-vanity) reaches its GPU through the Rust
 * trait `Backend` (src/gpu/mod.rs:41-52) and the CUDA entry points
 * `init_walk` / `walk` (src/gpu/kernel.cu:21-36).  The functions below are
 * what a Rust `Backend` implementation (or any other FFI) binds instead:
 * plain pointers and sizes, no CUDA or C++ types, errors returned as codes
 * with a message, never an abort.  One handle belongs to one host thread at a
 * time; there is no hidden global state.
 *
 * Packing conventions follow the reference:
 *   - public keys / u-coordinates: 8 little-endian uint32 words (32 LE bytes);
 *   - the Ed25519 public key: 8 big-endian words (mod.rs:110);
 *   - the name hash: 3 big-endian words, bytes 8-9 in the top half of the
 *     third word (mod.rs:113-117);
 *   - want / mask: 4 big-endian words of the destination hash (mod.rs:74-84);
 *   - a hit is (walker lane, walk index n): the identity is
 *     step_scalar(start[lane], n) || ed25519 seed (mod.rs:139-144).
 */
#ifndef LXMFV_H
#define LXMFV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes. */
#define LXMFV_OK 0
#define LXMFV_ERR_ARG -1     /* a bad argument (null pointer, size, range) */
#define LXMFV_ERR_CUDA -2    /* the CUDA runtime or driver reported an error */
#define LXMFV_ERR_NOMEM -3   /* a host or device allocation failed */
#define LXMFV_ERR_STATE -4   /* the call is not valid in the handle's state */
#define LXMFV_ERR_RECHECK -5 /* a GPU hit failed its from-scratch CPU recheck */
#define LXMFV_ERR_OVERFLOW -6 /* more hits than the caller's buffer holds */

typedef struct lxmfv_handle lxmfv_handle;

/* Walks.  Both visit the same keys k + 8n and give the same hashes and hits.
 * GROUP: affine additions of table points i*8B to a centre point, one batch
 *        inversion per group of `batch` keys (about half the field work).
 * XADD:  the reference's x-only differential addition (common.h:316-325)
 *        with Montgomery's batch inversion over `batch` keys. */
#define LXMFV_WALK_GROUP 0
#define LXMFV_WALK_XADD 1
#define LXMFV_MAX_HALF_GROUP 512

/* Option flags.  PHASE_SYNC (grouped walk, blocks of 256 or 512): a block
 * barrier after every group keeps a block's warps in the same phase of the
 * walk, so they share one phase's code in the instruction cache. */
#define LXMFV_FLAG_PHASE_SYNC 1u
/* REGCAP_80 (grouped walk, batch 256, block 256, with PHASE_SYNC): the kernel
 * built for three blocks per SM, at most 80 registers per thread and 24 warps
 * per SM, instead of two blocks at up to 128 registers (16 warps).  A point of
 * the autotuner's register-cap sweep. */
#define LXMFV_FLAG_REGCAP_80 2u
/* WARP_SPEC (grouped walk, batch 512 or 1024, block 0 or 768): each block's
 * warps split by role.  8 walker warps (32 lanes each, 256 lanes per block)
 * run the field arithmetic and hand every key's u through shared memory to 16
 * hash warps, which run the SHA-256 chain and the compare; the two phases of
 * the walk then overlap on the multiply-add and ALU pipes.  The same keys,
 * hashes and hits as the grouped walk.  Its waits are bounded: a launch whose
 * wait gave up fails at lxmfv_collect / lxmfv_launch with LXMFV_ERR_CUDA, and
 * the handle must be initialised again. */
#define LXMFV_FLAG_WARP_SPEC 4u

/* Opening options; zero fields take defaults.
 * Replaces the constants of src/gpu/cuda.rs:13-16 (BATCH, BLOCK,
 * THREADS_PER_SM) and CudaContext::new(0) (cuda.rs:33-64). */
typedef struct {
    int32_t device;       /* CUDA device ordinal */
    uint32_t lanes;       /* walker lanes (GPU threads); 0: one full wave of the device */
    uint32_t batch;       /* keys per inversion: XADD 16, 32, 64, 128; GROUP 32 .. 1024; 0: the fastest (GROUP 1024, XADD 128) */
    uint32_t block;       /* threads per block: 128, 256 or 512; 0: 512 with LXMFV_FLAG_PHASE_SYNC */
    uint32_t walk;        /* LXMFV_WALK_GROUP (0, default) or LXMFV_WALK_XADD */
    uint32_t flags;       /* LXMFV_FLAG_* */
    void* stream;         /* cudaStream_t to launch on; NULL: a stream of the handle's own */
} lxmfv_options;

/* One launch of the walk.  Mirrors LaunchArgs (src/gpu/mod.rs:29-38). */
typedef struct {
    uint32_t iters;        /* batches of B keys per lane in this launch */
    uint32_t ed[8];        /* Ed25519 public key, big-endian words */
    uint32_t name_hash[3]; /* name hash, big-endian words */
    uint32_t want[4];      /* destination-hash prefix, big-endian words */
    uint32_t mask[4];
    uint32_t q[8];         /* u(8B), little-endian words: the fixed step point */
    uint32_t max_hits;     /* hit slots filled at most (the reference uses 4096) */
    uint32_t dump_threads; /* lanes whose first dump_keys public keys are written */
    uint32_t dump_keys;    /* keys dumped per lane; 0: B (the reference's dump) */
} lxmfv_launch_args;

/* A hit: lane `thread` at walk index `n`.  The pair of src/gpu/cuda.rs:124-129. */
typedef struct {
    uint32_t thread;
    uint32_t reserved;
    uint64_t n;
} lxmfv_hit;

/* Opens device `opts->device`, builds the walker state for `lanes` lanes and
 * stores a handle in *out.  A handle is stored even on failure (when host
 * memory allows), so that lxmfv_last_error can say why; close it either way.
 * Replaces Cuda::new (src/gpu/cuda.rs:33-64). */
int lxmfv_open(const lxmfv_options* opts, lxmfv_handle** out);

/* The last error message of the handle ("" after success). */
const char* lxmfv_last_error(const lxmfv_handle* h);

/* "NVIDIA B200 (CUDA, compute 10.0, 148 SMs)"-style line.  Replaces
 * Backend::describe (mod.rs:43). Returns the full length (snprintf-style). */
int lxmfv_describe(const lxmfv_handle* h, char* buf, size_t len);

/* Walker lanes: Backend::threads (mod.rs:44). */
uint32_t lxmfv_threads(const lxmfv_handle* h);

/* Keys per batch inversion: Backend::batch (mod.rs:46). */
uint64_t lxmfv_batch(const lxmfv_handle* h);

/* The handle's walk (LXMFV_WALK_GROUP or LXMFV_WALK_XADD).  No counterpart in
 * the reference, which has the x-only walk only. */
uint32_t lxmfv_walk(const lxmfv_handle* h);

/* Sets every lane from u(k-8) and u(k): 16 little-endian words per lane,
 * n_words = 16 * lanes.  Walk indices restart at 0.  Replaces Backend::init
 * (mod.rs:48) / Cuda::init (cuda.rs:84-91) and the init_walk kernel
 * (kernel.cu:21-24). */
int lxmfv_init(lxmfv_handle* h, const uint32_t* u_prev_cur, size_t n_words);

/* Sets every lane from its start scalar k (32 little-endian bytes per lane,
 * n_bytes = 32 * lanes; clamped, with room to step, as random_start_scalar
 * makes them, main.rs:157-171) by a Montgomery ladder on the GPU.  Replaces
 * first_public_keys (mod.rs:212-228), which runs two X25519 per lane on the
 * CPU, followed by Backend::init. */
int lxmfv_init_from_scalars(lxmfv_handle* h, const uint8_t* scalars, size_t n_bytes);

/* u(k-8) and u(k) for `count` start scalars (32 LE bytes each, clamped with
 * room to step), computed on the GPU: 16 little-endian words per scalar into
 * u_prev_cur, the layout lxmfv_init takes.  Replaces first_public_keys
 * (mod.rs:212-228), which makes two X25519 per lane on the CPU.  Independent
 * of the handle's lanes and walker state. */
int lxmfv_first_public_keys(lxmfv_handle* h, const uint8_t* scalars, size_t count, uint32_t* u_prev_cur);

/* Runs one launch of the walk and waits for it: every lane walks
 * args->iters * B keys from where it stopped.  Writes up to `hits_cap` hits
 * to `hits` and their total count (which may exceed hits_cap and
 * args->max_hits) to *n_hits; when `dump` is not NULL, writes
 * dump_threads * dump_keys * 8 public-key words (lane-major), and when
 * `dump_addr` is not NULL, the matching 4-word destination hashes.
 * Replaces Backend::launch (mod.rs:50-51) / Cuda::launch (cuda.rs:93-132) and
 * the walk kernel (kernel.cu:26-36). */
int lxmfv_launch(lxmfv_handle* h, const lxmfv_launch_args* args, lxmfv_hit* hits, uint32_t hits_cap,
                 uint32_t* n_hits, uint32_t* dump, uint32_t* dump_addr);

/* The asynchronous half of lxmfv_launch: enqueues the walk on the handle's
 * stream and returns.  Hits accumulate on the device until lxmfv_collect.
 * No counterpart in the reference (its launch always synchronises,
 * cuda.rs:122); used to keep the walk back to back on the GPU. */
int lxmfv_launch_async(lxmfv_handle* h, const lxmfv_launch_args* args);

/* Waits for the handle's stream, copies back up to hits_cap hits (and the
 * dump of the last dumping launch), and clears the device hit queue. */
int lxmfv_collect(lxmfv_handle* h, lxmfv_hit* hits, uint32_t hits_cap, uint32_t* n_hits, uint32_t* dump,
                  uint32_t* dump_addr);

/* Device time of the last walk kernel, in milliseconds (CUDA events on the
 * launching stream; valid after lxmfv_launch or lxmfv_collect). */
float lxmfv_last_kernel_ms(const lxmfv_handle* h);

/* Releases the handle and its device memory (NULL is ignored). */
void lxmfv_close(lxmfv_handle* h);

/* ---- The search pool: many searches in one persistent kernel. ----
 * No counterpart in the reference, which runs one search per process
 * (GpuSearch, mod.rs:86-174) and starts more processes to search more
 * (fleet.sh).  Searches with different prefixes, aspects and identities are
 * admitted into a device-resident pool of walker lanes, walked together by a
 * persistent kernel that takes 32-lane chunks from a device work queue, and
 * retired as their hits come in.  Every step advances every active lane by
 * the same number of keys, so a search's hits do not depend on the rest of
 * the pool.  A step is a CUDA graph (reset, persistent kernel, hit read-back)
 * captured once per step length. */
typedef struct lxmfv_pool lxmfv_pool;

typedef struct {
    int32_t device;
    uint32_t capacity_lanes; /* walker lanes in the pool; 0: memory_budget / bytes per lane, else 2^20 */
    uint64_t memory_budget;  /* device bytes for lanes (108 per lane) when capacity_lanes is 0 */
    uint32_t batch;          /* keys per group: 64, 128, 256, 512 or 1024; 0: 1024 */
    uint32_t max_searches;   /* search slots; 0: 4096 */
    uint32_t max_hits;       /* hits held between polls; 0: 65536 */
    void* stream;            /* cudaStream_t; NULL: a stream of the pool's own */
} lxmfv_pool_options;

/* One search: the launch arguments' per-search fields (LaunchArgs,
 * mod.rs:29-38) and its number of lanes (a multiple of 32). */
typedef struct {
    uint32_t ed[8];
    uint32_t name_hash[3];
    uint32_t want[4];
    uint32_t mask[4];
    uint32_t lanes;
} lxmfv_search_desc;

/* A hit: search id, lane within the search, walk index.  The identity is
 * step_scalar(scalars[lane], n) || the search's Ed25519 seed. */
typedef struct {
    uint32_t search;
    uint32_t lane;
    uint64_t n;
} lxmfv_pool_hit;

typedef struct {
    uint32_t capacity_lanes, free_lanes, active_searches, active_lanes, batch, sms;
} lxmfv_pool_info_t;

int lxmfv_pool_open(const lxmfv_pool_options* opts, lxmfv_pool** out);
const char* lxmfv_pool_last_error(const lxmfv_pool* p);
int lxmfv_pool_info(const lxmfv_pool* p, lxmfv_pool_info_t* info);

/* Admits a search: `scalars` holds desc->lanes start scalars (32 LE bytes
 * each, clamped).  LXMFV_ERR_OVERFLOW when the pool has too few free lanes or
 * no free slot (admission against the memory budget). */
int lxmfv_pool_submit(lxmfv_pool* p, const lxmfv_search_desc* desc, const uint8_t* scalars, uint32_t* search_id);

/* Admits searches descs[0..n) in order, as many as fit: the longest prefix
 * for which the pool has free lanes and slots.  `scalars` holds every
 * search's start scalars back to back (descs[0].lanes of them, then
 * descs[1].lanes, ...).  Their start points run in one kernel, enqueued on
 * the pool's stream without waiting (lxmfv_pool_submit waits for each), so a
 * serving loop admits everything that arrived during a step at the cost of
 * one launch; the next step runs after it.  search_ids[i] receives the id of
 * descs[i] for i < *n_admitted.  LXMFV_ERR_OVERFLOW (nothing admitted) when
 * descs[0] does not fit; a CUDA error of the start kernel itself shows at the
 * next lxmfv_pool_poll. */
int lxmfv_pool_submit_many(lxmfv_pool* p, const lxmfv_search_desc* descs, uint32_t n, const uint8_t* scalars,
                           uint32_t* search_ids, uint32_t* n_admitted);

/* Frees a search's lanes; it takes no further part in steps. */
int lxmfv_pool_retire(lxmfv_pool* p, uint32_t search_id);

/* Enqueues one step: every active lane walks `groups` groups (groups *
 * batch keys).  Asynchronous. */
int lxmfv_pool_step(lxmfv_pool* p, uint32_t groups);

/* Waits for the enqueued steps and returns the hits found since the last
 * poll (up to cap; *n_hits is their total, which may exceed cap). */
int lxmfv_pool_poll(lxmfv_pool* p, lxmfv_pool_hit* hits, uint32_t cap, uint32_t* n_hits);

/* The walk index every lane of a search has reached (keys walked per lane). */
uint64_t lxmfv_pool_keys_per_lane(const lxmfv_pool* p, uint32_t search_id);

/* Device time of the last step in milliseconds (CUDA events). */
float lxmfv_pool_last_step_ms(const lxmfv_pool* p);

void lxmfv_pool_close(lxmfv_pool* p);

/* ---- Host helpers (CPU): the reference's address and scalar rules. ---- */

/* Prefix::parse (main.rs:206-216): 1..32 hex digits, any case; odd lengths
 * are padded with '0'.  Writes 16 prefix bytes and returns the nibble count,
 * or LXMFV_ERR_ARG. */
int lxmfv_prefix_parse(const char* text, uint8_t bytes[16]);

/* Prefix::matches (main.rs:218-224). */
int lxmfv_prefix_matches(const uint8_t bytes[16], int nibbles, const uint8_t address[16]);

/* prefix_words (mod.rs:74-84): big-endian want / mask words. */
void lxmfv_prefix_words(const uint8_t bytes[16], int nibbles, uint32_t want[4], uint32_t mask[4]);

/* name_hash (main.rs:174-176) of an aspect string, e.g. "lxmf.delivery". */
void lxmfv_name_hash(const char* aspect, uint8_t out[10]);

/* step_scalar (main.rs:125-137): k + 8n, little-endian. */
void lxmfv_step_scalar(const uint8_t k[32], uint64_t n, uint8_t out[32]);

/* previous_scalar (main.rs:140-152): k - 8. */
void lxmfv_previous_scalar(const uint8_t k[32], uint8_t out[32]);

/* Clamps k in place as random_start_scalar does (main.rs:161-163) and returns
 * 1 when it also passes its rejection rule (main.rs:164-169), else 0. */
int lxmfv_clamp_start(uint8_t k[32]);

/* Seeded draws: the ChaCha20 keystream (RFC 8439 block function; key = seed
 * as a u64 little-endian in bytes 0-7, zeros elsewhere; nonce 0; counter
 * from 0).  An identity is the first accepted 32-byte scalar draw followed by
 * the next 32 bytes (the Ed25519 seed); further scalars are further accepted
 * draws.  Returns the stream offset after the draws. */
uint64_t lxmfv_seeded_identity(uint64_t seed, uint8_t identity[64]);
uint64_t lxmfv_seeded_scalars(uint64_t seed, uint64_t offset, uint8_t* scalars, uint64_t count);

/* Fresh randomness from the operating system (getrandom), as the reference
 * draws it (main.rs:160, main.rs:294, mod.rs:103). */
int lxmfv_os_random(uint8_t* out, size_t len);

/* Ed25519 public key of a 32-byte seed (SigningKey::verifying_key). */
int lxmfv_ed25519_public(const uint8_t seed[32], uint8_t out[32]);

/* x25519(k, 9): the X25519 public key of a private key (clamps k). */
int lxmfv_x25519_base(const uint8_t k[32], uint8_t out[32]);

/* address_of_identity (main.rs:191-197), computed from scratch on the CPU with
 * an independent implementation (OpenSSL): the recheck every hit passes. */
int lxmfv_address_of_identity(const uint8_t identity[64], const uint8_t name_hash[10], uint8_t out[16]);

/* ---- The CPU search (the reference's default mode and the CPU half of
 * --gpu --cpu).  Runs only when called; no GPU entry point falls back to it. */

/* lxmfv_cpu_search found no hit before *stop became nonzero. */
#define LXMFV_STOPPED 1
#define LXMFV_CPU_MAX_THREADS 4096

/* lxmf_address (main.rs:180-189) on `count` 64-byte public keys (x_pub then
 * ed_pub) with one name hash, on this CPU thread: 16-byte outputs.  impl 0:
 * the fastest this CPU has (4, else 2, else 1); 1: portable C; 2: the x86 SHA
 * extensions; 3: the same, two keys at a time; 4: AVX-512F, sixteen keys at a
 * time, as the CPU search hashes them where the CPU has it (2 and 3:
 * LXMFV_ERR_STATE where the SHA extensions are absent, 4 where AVX-512F is). */
int lxmfv_cpu_addresses(const uint8_t* pks, uint64_t count, const uint8_t name_hash[10], uint8_t* out, int impl);

/* KeyWalk::next_batch (main.rs:255-289) from start scalar k: writes the
 * X25519 public keys u(k + 8n), n = 0 .. count-1, 32 bytes each.  It and
 * lxmfv_cpu_search walk on eight AVX-512 IFMA lanes where the CPU has them,
 * else in scalar 64-bit code; the environment variable LXMFV_CPU_WALK=scalar
 * or =ifma picks one (LXMFV_ERR_STATE where it is unavailable or unknown). */
int lxmfv_cpu_walk(const uint8_t start[32], uint64_t count, uint8_t* keys);

/* search on `threads` CPU threads (main.rs:292-323, fanned out as
 * run_search, main.rs:360-432) until one finds an address starting with the
 * prefix, or until *stop (read atomically) becomes nonzero.  seed NULL: each
 * thread draws its own start scalar and Ed25519 seed from the OS, as the
 * reference.  seed given: thread t walks seeded walker first_walker + t
 * (walker 0 = the seeded identity's scalar, walker w = the w-th further
 * scalar draw, first_walker <= 2^24) with the identity's Ed25519 seed.
 * *tries (may be NULL) is updated every 10 ms with the keys tried.  Writes
 * the rechecked 64-byte identity and returns LXMFV_OK; LXMFV_STOPPED when
 * stopped without a hit; LXMFV_ERR_RECHECK when a hit failed its recheck;
 * LXMFV_ERR_NOMEM when memory or threads ran out (threads already started are
 * stopped and joined first).
 * LXMFV_CPU_HASH=c, =ni or =x16 picks the SHA-256 code (portable C, the SHA
 * extensions, AVX-512F) instead of the fastest; LXMFV_ERR_STATE where the
 * CPU lacks it. */
int lxmfv_cpu_search(const uint8_t prefix[16], int nibbles, const uint8_t name_hash[10], int threads,
                     const uint64_t* seed, uint64_t first_walker, const int* stop, uint64_t* tries,
                     uint8_t identity[64]);

/* ---- Primitive kernels (the field and hash microbench). ---- */

/* Field op on `count` elements of 8 little-endian words on the GPU: inputs
 * drop bit 255 (fe_from_words, common.h:131-142), outputs are canonical
 * (fe_to_words, common.h:145-174).  op 0: a*b (fe_mul, common.h:75-89);
 * 1: a^2 (fe_sq, common.h:92-107); 2: a^(p-2) (fe_invert, common.h:115-128);
 * 3: batch inversion by Montgomery's trick over groups of `group` elements
 * (common.h:326-356).  Host buffers; returns LXMFV_OK. */
int lxmfv_fe_op(lxmfv_handle* h, int op, const uint32_t* a, const uint32_t* b, uint32_t* out, uint64_t count,
                uint32_t group);

/* ---- For callers that cannot allocate device memory. ---- */

/* Field elements the static scratch of lxmfv_fe_batch_invert_static holds:
 * the most a call may process (4 MiB of device memory, held on every GPU
 * that loads the library until the process exits). */
#define LXMFV_STATIC_SCRATCH_ELEMS 131072u

/* The batch inversion of lxmfv_fe_op op 3 on device buffers the caller owns,
 * with no device allocation: for callers that may not call cudaMalloc or
 * cudaFree (a host runtime that owns every device allocation and hands the
 * library its buffers, a loop that cannot take cudaFree's implicit device
 * synchronisation).  No counterpart in the reference.
 * d_a, d_out: device pointers on the current device, 16-byte aligned,
 * `count` elements of 8 little-endian words (inputs drop bit 255, outputs are
 * canonical); group 1..256.  d_out may equal d_a (in place); ranges that
 * overlap otherwise are rejected with LXMFV_ERR_ARG.  The kernel is enqueued
 * on `stream` (NULL: the default stream) and the call returns without
 * waiting for it.
 * The working storage is one static device array shared by every call:
 * count above LXMFV_STATIC_SCRATCH_ELEMS is rejected with LXMFV_ERR_ARG, and
 * calls whose kernels overlap on the GPU race on the array, so the caller
 * must order them.  The first call in a device's context looks up the
 * array's device address with that device current.  After cudaDeviceReset
 * the next call looks it up again.
 * A message for a non-zero return goes to err (err_len bytes) when given. */
int lxmfv_fe_batch_invert_static(const uint32_t* d_a, uint32_t* d_out, uint64_t count, uint32_t group, void* stream,
                                 char* err, size_t err_len);

/* The destination-hash chain on `count` 64-byte public keys (32 LE u bytes
 * then 32 key bytes) with one name hash: 16-byte outputs.  The three
 * compressions of lxmf_address (common.h:221-253).  Host buffers. */
int lxmfv_address_chain(lxmfv_handle* h, const uint8_t* pks, const uint8_t name_hash[10], uint8_t* out,
                        uint64_t count);

/* Integer-pipe throughput probe: runs `kind` on every SM for about `ms`
 * milliseconds and returns lane-operations per second in *ops_per_s.
 * Kinds: 0 mad.lo.u32, 1 mad.hi.u32, 2 xor + funnel shift, 3 mad.wide.u32
 * with a 64-bit addend, 4 add.u32, 5 mad.lo.u32 + xor (two pipes at once),
 * 6 funnel shift, 7 xor.  Diagnostic with no counterpart in the reference:
 * the denominators of the integer roofline. */
int lxmfv_peak_probe(lxmfv_handle* h, int kind, float ms, double* ops_per_s);

#ifdef __cplusplus
}
#endif

#endif /* LXMFV_H */
