// The CPU search: the reference's `lxmf-vanity <prefix>` mode and the CPU half
// of `--gpu --cpu` (search and KeyWalk, src/main.rs:230-323; run_search's
// thread fan-out, main.rs:360-432).  It runs only when a caller asks for a CPU
// search; the GPU entry points never fall back to it.
//
// Per thread, as the reference: one start scalar k and one Ed25519 seed; the
// X25519 keys u(k + 8n), 256 at a time, in walk order (the reference's
// KeyWalk uses x-only differential addition; here the grouped affine walk of
// the GPU kernels visits the same keys with a third of the field work); each
// key's address by the double SHA-256 (cpu_sha256.h: 16 keys at a time with
// AVX-512 where present, else the x86 SHA extensions, else portable C); the
// first match in walk order is rebuilt from its scalar and rechecked from
// scratch (OpenSSL) before it is returned.
// Field: GF(2^255-19) in 5 x 51-bit limbs with 128-bit products.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/lxmfv.h"
#include "cpu_sha256.h"

namespace {

typedef unsigned __int128 u128;
constexpr uint64_t MASK51 = (1ull << 51) - 1;
constexpr int BATCH = 256;  // keys per batch inversion (a group), as main.rs's BATCH
static_assert(BATCH % 16 == 0, "keys are hashed 16 at a time");

struct F {
    uint64_t l[5];
};

const F ONE = {{1, 0, 0, 0, 0}};

inline F carry(F a) {
    for (int i = 0; i < 4; i++) {
        a.l[i + 1] += a.l[i] >> 51;
        a.l[i] &= MASK51;
    }
    a.l[0] += 19 * (a.l[4] >> 51);
    a.l[4] &= MASK51;
    a.l[1] += a.l[0] >> 51;
    a.l[0] &= MASK51;
    return a;
}

inline F add(const F& a, const F& b) {
    F r;
    for (int i = 0; i < 5; i++) r.l[i] = a.l[i] + b.l[i];
    return carry(r);
}

// a - b + 4p: the limbs of a carried value stay below 2^52, 4p's are above.
inline F sub(const F& a, const F& b) {
    F r;
    r.l[0] = a.l[0] + 4 * (MASK51 - 18) - b.l[0];
    for (int i = 1; i < 5; i++) r.l[i] = a.l[i] + 4 * MASK51 - b.l[i];
    return carry(r);
}

inline F mul(const F& a, const F& b) {
    const uint64_t b1 = 19 * b.l[1], b2 = 19 * b.l[2], b3 = 19 * b.l[3], b4 = 19 * b.l[4];
    u128 t0 = (u128)a.l[0] * b.l[0] + (u128)a.l[1] * b4 + (u128)a.l[2] * b3 + (u128)a.l[3] * b2 + (u128)a.l[4] * b1;
    u128 t1 = (u128)a.l[0] * b.l[1] + (u128)a.l[1] * b.l[0] + (u128)a.l[2] * b4 + (u128)a.l[3] * b3 + (u128)a.l[4] * b2;
    u128 t2 = (u128)a.l[0] * b.l[2] + (u128)a.l[1] * b.l[1] + (u128)a.l[2] * b.l[0] + (u128)a.l[3] * b4 + (u128)a.l[4] * b3;
    u128 t3 = (u128)a.l[0] * b.l[3] + (u128)a.l[1] * b.l[2] + (u128)a.l[2] * b.l[1] + (u128)a.l[3] * b.l[0] + (u128)a.l[4] * b4;
    u128 t4 = (u128)a.l[0] * b.l[4] + (u128)a.l[1] * b.l[3] + (u128)a.l[2] * b.l[2] + (u128)a.l[3] * b.l[1] + (u128)a.l[4] * b.l[0];
    F r;
    t1 += (uint64_t)(t0 >> 51);
    r.l[0] = (uint64_t)t0 & MASK51;
    t2 += (uint64_t)(t1 >> 51);
    r.l[1] = (uint64_t)t1 & MASK51;
    t3 += (uint64_t)(t2 >> 51);
    r.l[2] = (uint64_t)t2 & MASK51;
    t4 += (uint64_t)(t3 >> 51);
    r.l[3] = (uint64_t)t3 & MASK51;
    r.l[4] = (uint64_t)t4 & MASK51;
    r.l[0] += 19 * (uint64_t)(t4 >> 51);
    r.l[1] += r.l[0] >> 51;
    r.l[0] &= MASK51;
    return r;
}

inline F sqr(const F& a) { return mul(a, a); }

inline F sqr_n(F x, int n) {
    for (int i = 0; i < n; i++) x = sqr(x);
    return x;
}

// z^(p-2) = z^(2^255 - 21) by the addition chain through z^(2^250 - 1).
F invert(const F& z) {
    const F z2 = sqr(z);
    const F z9 = mul(sqr_n(z2, 2), z);
    const F z11 = mul(z9, z2);
    const F e5 = mul(sqr(z11), z9);       // z^(2^5 - 1)
    const F e10 = mul(sqr_n(e5, 5), e5);  // z^(2^10 - 1)
    const F e20 = mul(sqr_n(e10, 10), e10);
    const F e40 = mul(sqr_n(e20, 20), e20);
    const F e50 = mul(sqr_n(e40, 10), e10);
    const F e100 = mul(sqr_n(e50, 50), e50);
    const F e200 = mul(sqr_n(e100, 100), e100);
    const F e250 = mul(sqr_n(e200, 50), e50);
    return mul(sqr_n(e250, 5), z11);  // z^(2^255 - 32 + 11)
}

// Little-endian bytes with bit 255 ignored (RFC 7748 decodeUCoordinate).
F from_bytes(const uint8_t b[32]) {
    uint64_t w[4];
    for (int i = 0; i < 4; i++) {
        w[i] = 0;
        for (int j = 7; j >= 0; j--) w[i] = (w[i] << 8) | b[8 * i + j];
    }
    w[3] &= 0x7fffffffffffffffull;
    F r;
    r.l[0] = w[0] & MASK51;
    r.l[1] = ((w[0] >> 51) | (w[1] << 13)) & MASK51;
    r.l[2] = ((w[1] >> 38) | (w[2] << 26)) & MASK51;
    r.l[3] = ((w[2] >> 25) | (w[3] << 39)) & MASK51;
    r.l[4] = w[3] >> 12;
    return r;
}

// The canonical encoding (the value mod p).
void to_bytes(uint8_t out[32], F a) {
    a = carry(carry(a));
    // Now a < 2^255 + 2^13; a >= p exactly when a + 19 carries out of bit 255.
    uint64_t q = (a.l[0] + 19) >> 51;
    for (int i = 1; i < 5; i++) q = (a.l[i] + q) >> 51;
    a.l[0] += 19 * q;
    for (int i = 0; i < 4; i++) {
        a.l[i + 1] += a.l[i] >> 51;
        a.l[i] &= MASK51;
    }
    a.l[4] &= MASK51;
    const uint64_t w[4] = {a.l[0] | (a.l[1] << 51), (a.l[1] >> 13) | (a.l[2] << 38), (a.l[2] >> 26) | (a.l[3] << 25),
                           (a.l[3] >> 39) | (a.l[4] << 12)};
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 8; j++) out[8 * i + j] = (uint8_t)(w[i] >> (8 * j));
}

// u(8B), little-endian.
const uint8_t U8B_BYTES[32] = {0x68, 0x99, 0xc9, 0x48, 0xed, 0x6f, 0x71, 0xf1, 0x1e, 0xa9, 0x74,
                               0xad, 0xca, 0xed, 0x78, 0x7a, 0xa1, 0x5c, 0xb6, 0xc8, 0x4d, 0x88,
                               0x3b, 0xd8, 0x2d, 0x5c, 0xd6, 0xaa, 0xd7, 0xa6, 0x5f, 0x27};

// v(8B), the even square root of u^3 + A u^2 + u at u = u(8B), little-endian 32-bit words.
const uint32_t V8B_WORDS[8] = {0x9f728718u, 0xc5296d6eu, 0x70c591f9u, 0x4f479c67u,
                               0x4066b08cu, 0x8dcf4469u, 0x8fb939e4u, 0x6085bbbau};

constexpr int HALF = BATCH / 2;  // M: a group is the 2M = BATCH keys around one centre

F from_words(const uint32_t w[8]) {
    uint8_t b[32];
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 4; j++) b[4 * i + j] = (uint8_t)(w[i] >> (8 * j));
    return from_bytes(b);
}

F small(uint64_t x) { return F{{x, 0, 0, 0, 0}}; }

// P1 + P2 on the Montgomery curve v^2 = u^3 + A u^2 + u (affine, P1 != +-P2).
void add_affine(const F& u1, const F& v1, const F& u2, const F& v2, F& u3, F& v3) {
    const F l = mul(sub(v2, v1), invert(sub(u2, u1)));
    u3 = sub(sub(sub(sqr(l), small(486662)), u1), u2);
    v3 = sub(mul(l, sub(u1, u3)), v1);
}

// The group table: T_i = i Q (i = 1..M) and T_0 = J = 2M Q, affine, with
// Q = 8B = (u(8B), v(8B)); built once by affine additions.
struct GroupTable {
    F u[HALF + 1], v[HALF + 1];
    GroupTable() {
        const F uq = from_bytes(U8B_BYTES), vq = from_words(V8B_WORDS);
        // T_2 = 2Q by the tangent: l = (3u^2 + 2Au + 1) / 2v.
        const F l = mul(add(add(mul(small(3), sqr(uq)), mul(small(2 * 486662), uq)), ONE), invert(add(vq, vq)));
        F tu = sub(sub(sqr(l), small(486662)), add(uq, uq));
        F tv = sub(mul(l, sub(uq, tu)), vq);
        u[1] = uq;
        v[1] = vq;
        u[2] = tu;
        v[2] = tv;
        for (int i = 3; i <= 2 * HALF; i++) {
            F nu, nv;
            add_affine(tu, tv, uq, vq, nu, nv);
            tu = nu;
            tv = nv;
            if (i <= HALF) {
                u[i] = tu;
                v[i] = tv;
            }
        }
        u[0] = tu;
        v[0] = tv;
    }
};

const GroupTable& group_table() {
    static const GroupTable t;  // thread-safe initialisation (C++11)
    return t;
}

// u(k + 8n) for n = 0, 1, 2, ... by the grouped affine walk, the same keys as
// KeyWalk (main.rs:230-290) with about a third of its field work: keys
// C - i Q and C + i Q share the denominator u_{iQ} - u_C, so one batch
// inversion over M + 1 denominators serves a whole group of 2M keys and the
// step to the next centre C + 2M Q.  Each group's keys come out in walk order.
struct Walk {
    F uc, vc;
    uint64_t next = 0;
    uint8_t buf[BATCH][32];

    int init(const uint8_t k[32]) {
        // y of P = kB = (k/8) Q from u(k - 8) and u(k) (Okeya-Sakurai recovery
        // with -Q, since P - Q is the known neighbour), then C = P + M Q.
        uint8_t prev[32], b[32];
        lxmfv_previous_scalar(k, prev);
        if (lxmfv_x25519_base(prev, b) != LXMFV_OK) return LXMFV_ERR_STATE;
        const F um8 = from_bytes(b);
        if (lxmfv_x25519_base(k, b) != LXMFV_OK) return LXMFV_ERR_STATE;
        const F uk = from_bytes(b);
        const F xp = from_bytes(U8B_BYTES), yp = sub(F{{0, 0, 0, 0, 0}}, from_words(V8B_WORDS));
        // recover_y with (X1:Z1) = (uk:1), (X2:Z2) = (um8:1)
        F v1 = xp;
        F v2 = add(uk, v1);
        F v3 = sub(uk, v1);
        v3 = mul(sqr(v3), um8);
        v1 = small(2 * 486662);
        v2 = add(v2, v1);
        const F v4 = add(mul(xp, uk), ONE);
        v2 = mul(v2, v4);
        v2 = sub(v2, v1);
        const F Y = sub(v2, v3);
        const F c = add(yp, yp);
        const F zi = invert(c);
        const F pu = uk, pv = mul(Y, zi);  // X = c uk, Z = c: u = uk
        const GroupTable& t = group_table();
        add_affine(pu, pv, t.u[HALF], t.v[HALF], uc, vc);
        next = 0;
        return LXMFV_OK;
    }

    // The group of keys next .. next + BATCH - 1 into buf, in walk order.
    void group() {
        const GroupTable& t = group_table();
        F pre[HALF + 1];
        F acc = sub(t.u[0], uc);
        for (int i = 1; i <= HALF; i++) {
            pre[i] = acc;
            acc = mul(acc, sub(t.u[i], uc));
        }
        F inv = invert(acc);
        const F s0 = add(uc, small(486662));
        F vnext = vc, unext = uc;
        for (int i = HALF; i >= 0; i--) {
            F invi = inv;  // 1 / (u_{T_i} - u_C)
            if (i > 0) {
                invi = mul(inv, pre[i]);
                inv = mul(inv, sub(t.u[i], uc));
            }
            const F sum = add(s0, t.u[i]);
            const F lp = mul(sub(t.v[i], vc), invi);
            const F up = sub(sqr(lp), sum);  // C + T_i (i = 0: the next centre C + J)
            if (i > 0) {
                const F lm = mul(add(t.v[i], vc), invi);
                to_bytes(buf[HALF - i], sub(sqr(lm), sum));  // C - T_i: key c - i
                if (i < HALF) to_bytes(buf[HALF + i], up);    // C + T_i: key c + i
            } else {
                to_bytes(buf[HALF], uc);  // the centre: key c
                vnext = sub(mul(lp, sub(uc, up)), vc);
                unext = up;
            }
        }
        uc = unext;
        vc = vnext;
    }

    // The next `len` <= BATCH keys (a whole group; a shorter request keeps its
    // first keys and ends the walk); returns the walk index of the first.
    uint64_t batch(uint8_t (*out)[32], int len) {
        group();
        memcpy(out, buf, 32 * (size_t)len);
        const uint64_t first = next;
        next += BATCH;
        return first;
    }
};

struct Shared {
    const uint8_t* prefix;
    int nibbles;
    const uint8_t* nh;
    const int* stop;
    std::atomic<uint64_t> tries{0};
    std::atomic<int> found{0}, error{0};
    uint8_t* identity_out;
};

inline bool stopped(const Shared& s) {
    return __atomic_load_n(s.stop, __ATOMIC_RELAXED) != 0 || s.found.load(std::memory_order_relaxed) != 0 ||
           s.error.load(std::memory_order_relaxed) != 0;
}

// How a walker hashes: portable C, the SHA extensions two keys at a time, or
// AVX-512 sixteen keys at a time.
enum Hasher { HASH_C, HASH_NI, HASH_X16 };

// The addresses of two public keys.
template <Hasher H>
inline void hash_pair(uint8_t pk[2][64], uint8_t blocks[2][64], uint8_t h[2][16]) {
#if defined(__x86_64__)
    if (H == HASH_NI) {
        cpu_sha::address2_ni(pk[0], pk[1], blocks, h[0], h[1]);
        return;
    }
#endif
    cpu_sha::address<false>(pk[0], blocks[0], h[0]);
    cpu_sha::address<false>(pk[1], blocks[1], h[1]);
}

// Bit m set where key first + m of `keys` (16 of them) matches the prefix.
inline uint32_t match16(const uint8_t (*keys)[32], const uint8_t* ed_pub, const uint8_t* nh, const uint32_t want[4],
                        const uint32_t mask[4]) {
#if defined(__x86_64__)
    return cpu_sha::x16::match16(keys[0], 32, ed_pub, nh, want, mask);
#else
    (void)keys, (void)ed_pub, (void)nh, (void)want, (void)mask;
    return 0;
#endif
}

// One walker: search (main.rs:292-323) from scalar `start` with Ed25519 seed `ed_seed`.
template <Hasher H>
void walker(Shared* s, const uint8_t* start, const uint8_t* ed_seed) {
    uint8_t ed_pub[32];
    Walk w;
    if (lxmfv_ed25519_public(ed_seed, ed_pub) != LXMFV_OK || w.init(start) != LXMFV_OK) {
        s->error.store(LXMFV_ERR_STATE);
        return;
    }
    std::vector<uint8_t> keybuf(BATCH * 32);
    uint8_t(*keys)[32] = reinterpret_cast<uint8_t(*)[32]>(keybuf.data());
    uint8_t pk[2][64], blocks[2][64], h[2][16];
    for (int j = 0; j < 2; j++) {
        memcpy(pk[j] + 32, ed_pub, 32);
        cpu_sha::address_block(s->nh, blocks[j]);
    }
    uint32_t want[4], mask[4];
    lxmfv_prefix_words(s->prefix, s->nibbles, want, mask);
    while (!stopped(*s)) {
        const uint64_t first = w.batch(keys, BATCH);
        uint32_t hits16 = 0;
        for (int i = 0; i < BATCH; i++) {
            // Keys are hashed sixteen at a time (AVX-512: a bit per matching
            // key) or in pairs (two SHA-256 streams interleaved where the CPU
            // has the SHA extensions), and checked in walk order.
            if (H == HASH_X16) {
                if ((i & 15) == 0) hits16 = match16(keys + i, ed_pub, s->nh, want, mask);
                if (!(hits16 >> (i & 15) & 1)) {
                    if (!(hits16 >> (i & 15))) i |= 15;  // no match left in these 16
                    continue;
                }
            } else {
                if ((i & 1) == 0) {
                    memcpy(pk[0], keys[i], 32);
                    memcpy(pk[1], keys[i + 1], 32);
                    hash_pair<H>(pk, blocks, h);
                }
                if (!lxmfv_prefix_matches(s->prefix, s->nibbles, h[i & 1])) continue;
            }
            uint8_t ident[64], addr[16];
            lxmfv_step_scalar(start, first + (uint64_t)i, ident);
            memcpy(ident + 32, ed_seed, 32);
            // Recompute from scratch: never hand back a key the fast path got wrong.
            if (lxmfv_address_of_identity(ident, s->nh, addr) != LXMFV_OK ||
                !lxmfv_prefix_matches(s->prefix, s->nibbles, addr)) {
                s->error.store(LXMFV_ERR_RECHECK);
                return;
            }
            int expected = 0;
            if (s->found.compare_exchange_strong(expected, 1)) memcpy(s->identity_out, ident, 64);
            s->tries.fetch_add((uint64_t)i + 1, std::memory_order_relaxed);
            return;
        }
        s->tries.fetch_add(BATCH, std::memory_order_relaxed);
    }
}

bool use_sha_ni() {
#if defined(__x86_64__)
    return cpu_sha::have_sha_ni();
#else
    return false;
#endif
}

bool use_x16() {
#if defined(__x86_64__)
    return cpu_sha::x16::available();
#else
    return false;
#endif
}

}  // namespace

extern "C" int lxmfv_cpu_addresses(const uint8_t* pks, uint64_t count, const uint8_t name_hash[10], uint8_t* out,
                                   int impl) {
    if ((count && (!pks || !out)) || !name_hash || impl < 0 || impl > 4) return LXMFV_ERR_ARG;
    if ((impl == 2 || impl == 3) && !use_sha_ni()) return LXMFV_ERR_STATE;
    if (impl == 4 && !use_x16()) return LXMFV_ERR_STATE;
    if (impl == 0 && use_x16()) impl = 4;
#if defined(__x86_64__)
    if (impl == 4) {
        uint64_t i = 0;
        for (; i + 16 <= count; i += 16)
            cpu_sha::x16::address16_bytes(pks + 64 * i, 64, pks + 64 * i + 32, 64, name_hash, out + 16 * i);
        if (i < count) {
            // The last keys, padded to 16 with copies of the final one.
            uint8_t tail[16][64], addrs[16][16];
            for (int m = 0; m < 16; m++) memcpy(tail[m], pks + 64 * std::min<uint64_t>(i + m, count - 1), 64);
            cpu_sha::x16::address16_bytes(tail[0], 64, tail[0] + 32, 64, name_hash, addrs[0]);
            memcpy(out + 16 * i, addrs, 16 * (size_t)(count - i));
        }
        return LXMFV_OK;
    }
    if (impl == 3) {
        uint8_t blocks[2][64];
        cpu_sha::address_block(name_hash, blocks[0]);
        cpu_sha::address_block(name_hash, blocks[1]);
        uint64_t i = 0;
        for (; i + 1 < count; i += 2)
            cpu_sha::address2_ni(pks + 64 * i, pks + 64 * (i + 1), blocks, out + 16 * i, out + 16 * (i + 1));
        if (i < count) cpu_sha::address<true>(pks + 64 * i, blocks[0], out + 16 * i);
        return LXMFV_OK;
    }
#endif
    const bool ni = impl == 2 || (impl == 0 && use_sha_ni());
    uint8_t block[64];
    cpu_sha::address_block(name_hash, block);
    for (uint64_t i = 0; i < count; i++) {
        if (ni)
            cpu_sha::address<true>(pks + 64 * i, block, out + 16 * i);
        else
            cpu_sha::address<false>(pks + 64 * i, block, out + 16 * i);
    }
    return LXMFV_OK;
}

extern "C" int lxmfv_cpu_walk(const uint8_t start[32], uint64_t count, uint8_t* keys) {
    if (!start || (count && !keys)) return LXMFV_ERR_ARG;
    Walk w;
    if (w.init(start) != LXMFV_OK) return LXMFV_ERR_STATE;
    std::vector<uint8_t> tmp(BATCH * 32);
    for (uint64_t done = 0; done < count;) {
        const int len = (int)std::min<uint64_t>(BATCH, count - done);
        w.batch(reinterpret_cast<uint8_t(*)[32]>(tmp.data()), len);
        memcpy(keys + 32 * done, tmp.data(), 32 * (size_t)len);
        done += (uint64_t)len;
    }
    return LXMFV_OK;
}

extern "C" int lxmfv_cpu_search(const uint8_t prefix[16], int nibbles, const uint8_t name_hash[10], int threads,
                                const uint64_t* seed, uint64_t first_walker, const int* stop, uint64_t* tries,
                                uint8_t identity[64]) {
    if (!prefix || nibbles < 1 || nibbles > 32 || !name_hash || threads < 1 || threads > LXMFV_CPU_MAX_THREADS ||
        !stop || !identity)
        return LXMFV_ERR_ARG;
    if (!seed && first_walker) return LXMFV_ERR_ARG;
    if (seed && first_walker > (1ull << 24)) return LXMFV_ERR_ARG;
    // Start scalars and Ed25519 seeds, 32 bytes each per thread.
    std::vector<uint8_t> starts(32 * (size_t)threads), eds(32 * (size_t)threads);
    if (seed) {
        // Walker w of the seeded stream: w = 0 starts at the identity's own
        // scalar, w >= 1 at the w-th further draw; all share the identity's
        // Ed25519 seed.  The GPU's seeded lanes use the same numbering.
        uint8_t ident[64];
        uint64_t off = lxmfv_seeded_identity(*seed, ident);
        // Draws 1 .. last come from the stream in order; only this call's
        // walkers are kept, so memory stays at one chunk whatever first_walker.
        const uint64_t last = first_walker + (uint64_t)threads - 1;
        constexpr uint64_t CHUNK = 4096;
        std::vector<uint8_t> chunk(32 * CHUNK);
        for (uint64_t done = 0; done < last;) {
            const uint64_t n = std::min(CHUNK, last - done);
            off = lxmfv_seeded_scalars(*seed, off, chunk.data(), n);
            for (uint64_t i = 0; i < n; i++) {
                const uint64_t wk = done + i + 1;
                if (wk >= first_walker) memcpy(&starts[32 * (size_t)(wk - first_walker)], &chunk[32 * i], 32);
            }
            done += n;
        }
        if (first_walker == 0) memcpy(&starts[0], ident, 32);
        for (int t = 0; t < threads; t++) memcpy(&eds[32 * (size_t)t], ident + 32, 32);
    } else {
        // As the reference: each thread its own random scalar and Ed25519 seed.
        for (int t = 0; t < threads; t++) {
            uint8_t* k = &starts[32 * (size_t)t];
            do {
                if (lxmfv_os_random(k, 32) != LXMFV_OK) return LXMFV_ERR_STATE;
            } while (!lxmfv_clamp_start(k));
            if (lxmfv_os_random(&eds[32 * (size_t)t], 32) != LXMFV_OK) return LXMFV_ERR_STATE;
        }
    }
    Shared s;
    s.prefix = prefix;
    s.nibbles = nibbles;
    s.nh = name_hash;
    s.stop = stop;
    s.identity_out = identity;
    std::vector<std::thread> pool;
    pool.reserve((size_t)threads);
    // The fastest hasher this CPU has; LXMFV_CPU_HASH=c|ni|x16 picks one (tests
    // run each), LXMFV_ERR_STATE where the CPU lacks it.
    void (*run)(Shared*, const uint8_t*, const uint8_t*) =
        use_x16() ? walker<HASH_X16> : use_sha_ni() ? walker<HASH_NI> : walker<HASH_C>;
    if (const char* force = getenv("LXMFV_CPU_HASH")) {
        if (!strcmp(force, "c"))
            run = walker<HASH_C>;
        else if (!strcmp(force, "ni") && use_sha_ni())
            run = walker<HASH_NI>;
        else if (!strcmp(force, "x16") && use_x16())
            run = walker<HASH_X16>;
        else
            return LXMFV_ERR_STATE;
    }
    for (int t = 0; t < threads; t++) pool.emplace_back(run, &s, &starts[32 * (size_t)t], &eds[32 * (size_t)t]);
    while (!stopped(s)) {
        if (tries) __atomic_store_n(tries, s.tries.load(std::memory_order_relaxed), __ATOMIC_RELAXED);
        std::this_thread::sleep_for(std::chrono::milliseconds(10));
    }
    for (auto& th : pool) th.join();
    if (tries) __atomic_store_n(tries, s.tries.load(), __ATOMIC_RELAXED);
    if (s.error.load()) return s.error.load();
    return s.found.load() ? LXMFV_OK : LXMFV_STOPPED;
}
