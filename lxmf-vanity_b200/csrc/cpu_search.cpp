// The CPU search: the reference's `lxmf-vanity <prefix>` mode and the CPU half
// of `--gpu --cpu` (search and KeyWalk, src/main.rs:230-323; run_search's
// thread fan-out, main.rs:360-432).  It runs only when a caller asks for a CPU
// search; the GPU entry points never fall back to it.
//
// Per thread, as the reference: one start scalar k and one Ed25519 seed; the
// X25519 keys u(k + 8n) in walk order, a group at a time (the reference's
// KeyWalk uses x-only differential addition; here the grouped affine walk of
// the GPU kernels visits the same keys with a third of the field work: 2048
// keys per group on eight AVX-512 IFMA lanes where the CPU has them, else 256
// per group in scalar code); each
// key's address by the double SHA-256 (cpu_sha256.h: 16 keys at a time with
// AVX-512 where present, else the x86 SHA extensions, else portable C); the
// first match in walk order is rebuilt from its scalar and rechecked from
// scratch (OpenSSL) before it is returned.
// Field: GF(2^255-19) in 5 x 51-bit limbs, with 128-bit products (scalar) or
// 52-bit multiply-adds (IFMA lanes).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
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
template <int M>
struct GroupTable {
    F u[M + 1], v[M + 1];
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
        for (int i = 3; i <= 2 * M; i++) {
            F nu, nv;
            add_affine(tu, tv, uq, vq, nu, nv);
            tu = nu;
            tv = nv;
            if (i <= M) {
                u[i] = tu;
                v[i] = tv;
            }
        }
        u[0] = tu;
        v[0] = tv;
    }
};

template <int M>
const GroupTable<M>& group_table() {
    static const GroupTable<M> t;  // thread-safe initialisation (C++11)
    return t;
}

// P = kB in affine coordinates from u(k - 8) and u(k): Okeya-Sakurai y
// recovery with -Q, since P - Q is the known neighbour.
int start_point(const uint8_t k[32], F& pu, F& pv) {
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
    pu = uk;
    pv = mul(Y, zi);  // X = c uk, Z = c: u = uk
    return LXMFV_OK;
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

    static constexpr int SIZE = BATCH;

    // The walk from scalar k: the first group's centre C = P + M Q.
    int init(const uint8_t k[32]) {
        F pu, pv;
        if (int rc = start_point(k, pu, pv)) return rc;
        const GroupTable<HALF>& t = group_table<HALF>();
        add_affine(pu, pv, t.u[HALF], t.v[HALF], uc, vc);
        next = 0;
        return LXMFV_OK;
    }

    // The group of keys next .. next + BATCH - 1 into buf, in walk order.
    void group() {
        const GroupTable<HALF>& t = group_table<HALF>();
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

    // The next group; *first: the walk index of its first key.
    void advance(uint64_t* first) {
        group();
        *first = next;
        next += SIZE;
    }

    // The group's keys as 32-byte rows in walk order.
    const uint8_t (*keys())[32] { return buf; }

    // Bit m set where key i + m of the group matches (i a multiple of 16).
    uint32_t match16(int i, const cpu_sha::Shared16& shared, const uint32_t want[4], const uint32_t mask[4]) const {
#if defined(__x86_64__)
        return cpu_sha::x16::match16_shared(buf[i], 32, shared, want, mask);
#else
        (void)i, (void)shared, (void)want, (void)mask;
        return 0;
#endif
    }
};

#if defined(__x86_64__)
// The same walk with the field work on eight lanes of AVX-512 IFMA (52-bit
// multiply-add): GF(2^255-19) in the same 5 x 51-bit limbs, one walker's
// group elements spread over the lanes.  Groups are 2048 keys (M = 1024), so
// that the one scalar inversion per group costs about 1/8 of a multiply per
// key.
namespace ifma {

#define LXCPU_IFMA __attribute__((target("avx512f,avx512ifma")))

constexpr int M = 1024;      // a group is the 2M keys around one centre
constexpr int ROWS = M / 8;  // group elements per lane: lane j holds i = 1 + j + 8r

// Eight field elements, limb-major: l[k] holds limb k of lanes 0..7.  Every
// operation returns limbs below 2^52 (the multiplier reads 52 bits).
struct alignas(64) Lanes {
    uint64_t l[5][8];
};

struct Table {
    Lanes u[ROWS], v[ROWS];  // T_i = iQ, i = 1..M, lane-major
    F u0, v0, uM, vM;        // T_0 = J = 2M Q and T_M
    Table() {
        const GroupTable<M>& t = group_table<M>();
        for (int r = 0; r < ROWS; r++)
            for (int j = 0; j < 8; j++)
                for (int k = 0; k < 5; k++) {
                    u[r].l[k][j] = t.u[1 + j + 8 * r].l[k];
                    v[r].l[k][j] = t.v[1 + j + 8 * r].l[k];
                }
        u0 = t.u[0];
        v0 = t.v[0];
        uM = t.u[M];
        vM = t.v[M];
    }
};

const Table& table() {
    static const Table t;
    return t;
}

typedef __m512i V;
struct FV {
    V l[5];
};

LXCPU_IFMA inline FV load(const Lanes& a) {
    FV r;
    for (int k = 0; k < 5; k++) r.l[k] = _mm512_load_si512((const void*)a.l[k]);
    return r;
}
LXCPU_IFMA inline void store(Lanes& a, const FV& x) {
    for (int k = 0; k < 5; k++) _mm512_store_si512((void*)a.l[k], x.l[k]);
}
LXCPU_IFMA inline FV bcast(const F& a) {
    FV r;
    for (int k = 0; k < 5; k++) r.l[k] = _mm512_set1_epi64((long long)a.l[k]);
    return r;
}
LXCPU_IFMA inline V times19(V x) { return _mm512_add_epi64(_mm512_add_epi64(_mm512_slli_epi64(x, 4), _mm512_slli_epi64(x, 1)), x); }

// One carry step on every limb at once (no ripple): limbs below 2^63 in;
// limb i keeps its low 51 bits plus limb i-1's carry (limb 0: 19 times limb
// 4's), so below 2^51 + 2^17 out, inside the multiplier's 52 bits.
LXCPU_IFMA inline FV carry(FV a) {
    const V m = _mm512_set1_epi64((long long)MASK51);
    V c[5];
    for (int i = 0; i < 5; i++) c[i] = _mm512_srli_epi64(a.l[i], 51);
    for (int i = 0; i < 5; i++) a.l[i] = _mm512_and_si512(a.l[i], m);
    a.l[0] = _mm512_add_epi64(a.l[0], times19(c[4]));
    for (int i = 1; i < 5; i++) a.l[i] = _mm512_add_epi64(a.l[i], c[i - 1]);
    return a;
}

// a + b without the carry: limbs below 2^52 + 2^18, fit only for sub's b.
LXCPU_IFMA inline FV add_loose(const FV& a, const FV& b) {
    FV r;
    for (int k = 0; k < 5; k++) r.l[k] = _mm512_add_epi64(a.l[k], b.l[k]);
    return r;
}

LXCPU_IFMA inline FV add(const FV& a, const FV& b) { return carry(add_loose(a, b)); }

// a - b + 4p without the carry (b's limbs at most 4p's, about 2^53): limbs
// below 2^54, fit only for to_words (which carries first) or carry().
LXCPU_IFMA inline FV sub_loose(const FV& a, const FV& b) {
    FV r;
    r.l[0] = _mm512_sub_epi64(_mm512_add_epi64(a.l[0], _mm512_set1_epi64((long long)(4 * (MASK51 - 18)))), b.l[0]);
    for (int k = 1; k < 5; k++)
        r.l[k] = _mm512_sub_epi64(_mm512_add_epi64(a.l[k], _mm512_set1_epi64((long long)(4 * MASK51))), b.l[k]);
    return r;
}

// a - b + 4p, as the scalar sub.
LXCPU_IFMA inline FV sub(const FV& a, const FV& b) { return carry(sub_loose(a, b)); }

// a * b mod p.  A 52 x 52-bit product splits at bit 52: its low half goes to
// column i + j and its high half, worth 2^52 = 2 * 2^51, to column i + j + 1
// doubled.  Columns are built one at a time (its low halves, then the high
// halves from the column below, doubled), so that few accumulators are live;
// columns 5..9 fold down with 2^255 = 19.  Column bounds: 5 low + 10 high
// halves < 2^56; after the fold below 2^62.
LXCPU_IFMA inline FV mul(const FV& a, const FV& b) {
    V z[10];
#pragma GCC unroll 10
    for (int k = 0; k < 10; k++) {
        V lo = _mm512_setzero_si512(), hi = _mm512_setzero_si512();
#pragma GCC unroll 5
        for (int i = 0; i < 5; i++) {
            if (k - i >= 0 && k - i < 5) lo = _mm512_madd52lo_epu64(lo, a.l[i], b.l[k - i]);
            if (k - 1 - i >= 0 && k - 1 - i < 5) hi = _mm512_madd52hi_epu64(hi, a.l[i], b.l[k - 1 - i]);
        }
        z[k] = _mm512_add_epi64(lo, _mm512_slli_epi64(hi, 1));
    }
    FV r;
    for (int k = 0; k < 5; k++) r.l[k] = _mm512_add_epi64(z[k], times19(z[k + 5]));
    return carry(r);
}

// a^2, column by column: the squares once and the cross products once,
// doubled (column k = lo + 2 hi of the squares, 2 lo + 4 hi of the cross
// products).
LXCPU_IFMA inline FV sqr(const FV& a) {
    V z[10];
#pragma GCC unroll 10
    for (int k = 0; k < 10; k++) {
        V sq = _mm512_setzero_si512(), cr = _mm512_setzero_si512();
        if ((k & 1) == 0 && k / 2 < 5) sq = _mm512_madd52lo_epu64(sq, a.l[k / 2], a.l[k / 2]);
        if ((k & 1) == 1 && (k - 1) / 2 < 5)
            sq = _mm512_add_epi64(sq, _mm512_slli_epi64(
                                          _mm512_madd52hi_epu64(_mm512_setzero_si512(), a.l[(k - 1) / 2], a.l[(k - 1) / 2]), 1));
        V xl = _mm512_setzero_si512(), xh = _mm512_setzero_si512();
#pragma GCC unroll 5
        for (int i = 0; i < 5; i++) {
            const int j = k - i, jh = k - 1 - i;
            if (j > i && j < 5) xl = _mm512_madd52lo_epu64(xl, a.l[i], a.l[j]);
            if (jh > i && jh < 5) xh = _mm512_madd52hi_epu64(xh, a.l[i], a.l[jh]);
        }
        cr = _mm512_add_epi64(_mm512_slli_epi64(xl, 1), _mm512_slli_epi64(xh, 2));
        z[k] = _mm512_add_epi64(sq, cr);
    }
    FV r;
    for (int k = 0; k < 5; k++) r.l[k] = _mm512_add_epi64(z[k], times19(z[k + 5]));
    return carry(r);
}

// The canonical encodings of the eight lanes as four little-endian 64-bit
// words each (w[i] lane j), as the scalar to_bytes.  Limbs below 2^63 in: one
// carry leaves a value below 2^255 + 2^222 < 2p, where q = [a >= p] is the
// carry out of a + 19 (rippled through the limbs); the last pass ripples.
LXCPU_IFMA inline void to_words(FV a, V w[4]) {
    a = carry(a);
    const V m = _mm512_set1_epi64((long long)MASK51);
    V q = _mm512_srli_epi64(_mm512_add_epi64(a.l[0], _mm512_set1_epi64(19)), 51);
    for (int i = 1; i < 5; i++) q = _mm512_srli_epi64(_mm512_add_epi64(a.l[i], q), 51);
    a.l[0] = _mm512_add_epi64(a.l[0], times19(q));
    for (int i = 0; i < 4; i++) {
        a.l[i + 1] = _mm512_add_epi64(a.l[i + 1], _mm512_srli_epi64(a.l[i], 51));
        a.l[i] = _mm512_and_si512(a.l[i], m);
    }
    a.l[4] = _mm512_and_si512(a.l[4], m);
    w[0] = _mm512_or_si512(a.l[0], _mm512_slli_epi64(a.l[1], 51));
    w[1] = _mm512_or_si512(_mm512_srli_epi64(a.l[1], 13), _mm512_slli_epi64(a.l[2], 38));
    w[2] = _mm512_or_si512(_mm512_srli_epi64(a.l[2], 26), _mm512_slli_epi64(a.l[3], 25));
    w[3] = _mm512_or_si512(_mm512_srli_epi64(a.l[3], 39), _mm512_slli_epi64(a.l[4], 12));
}

// Keys are stored word-major: words[j][k] is 32-bit word j (little-endian)
// of key k of the group, so that sixteen keys' word j is one vector load for
// the hasher.  STRIDE leaves room past the last key for a full store.
constexpr int STRIDE = 2 * M + 16;

// The eight lanes' encodings into keys base .. base + 7 of words (lane j to
// key base + j, or to base + 7 - j when `reverse`).
LXCPU_IFMA inline void store_words(const FV& a, uint32_t (*words)[STRIDE], int base, bool reverse) {
    V w[4];
    to_words(a, w);
    const __m256i rev = _mm256_set_epi32(0, 1, 2, 3, 4, 5, 6, 7);
    for (int i = 0; i < 4; i++) {
        __m256i lo = _mm512_cvtepi64_epi32(w[i]);
        __m256i hi = _mm512_cvtepi64_epi32(_mm512_srli_epi64(w[i], 32));
        if (reverse) {
            lo = _mm256_permutevar8x32_epi32(lo, rev);
            hi = _mm256_permutevar8x32_epi32(hi, rev);
        }
        _mm256_storeu_si256((__m256i*)(words[2 * i] + base), lo);
        _mm256_storeu_si256((__m256i*)(words[2 * i + 1] + base), hi);
    }
}

struct Scratch {
    Lanes pre[ROWS];  // lane j, row r: the product of its elements before row r
    Lanes acc;
    alignas(64) uint32_t words[8][STRIDE];
    uint8_t buf[2 * M][32];  // the same keys as bytes, filled on request
};

// One group: scratch->words gets keys c - M .. c + M - 1 in walk order, and
// (uc, vc) moves to the next centre C + J.  The denominators u_{T_i} - u_C,
// i = 1..M, are eight interleaved Montgomery chains (one per lane); their
// eight totals and T_0's denominator share one scalar inversion.
LXCPU_IFMA void group(F& uc, F& vc, Scratch* s) {
    const Table& t = table();
    const FV UC = bcast(uc), VC = bcast(vc);
    FV acc = bcast(ONE);
    for (int r = 0; r < ROWS; r++) {
        store(s->pre[r], acc);
        acc = mul(acc, sub(load(t.u[r]), UC));
    }
    store(s->acc, acc);
    // Scalar: d0 = u_J - u_C and the eight lane totals, inverted together.
    F q[9], run[9];
    q[0] = ::sub(t.u0, uc);
    for (int j = 0; j < 8; j++)
        for (int k = 0; k < 5; k++) q[1 + j].l[k] = s->acc.l[k][j];
    run[0] = q[0];
    for (int m = 1; m < 9; m++) run[m] = ::mul(run[m - 1], q[m]);
    F inv = invert(run[8]);
    Lanes lane_inv;
    for (int m = 8; m >= 1; m--) {
        const F x = ::mul(inv, run[m - 1]);  // 1 / q[m]
        for (int k = 0; k < 5; k++) lane_inv.l[k][m - 1] = x.l[k];
        inv = ::mul(inv, q[m]);
    }
    const F inv_d0 = inv;
    const F s0 = ::add(uc, small(486662));
    const FV S0 = bcast(s0);
    FV INV = load(lane_inv);
    for (int r = ROWS - 1; r >= 0; r--) {
        const FV TU = load(t.u[r]), TV = load(t.v[r]);
        const FV invi = mul(INV, load(s->pre[r]));  // 1 / (u_{T_i} - u_C)
        INV = mul(INV, sub(TU, UC));
        const FV sum = add_loose(S0, TU);  // only ever subtracted
        const FV lp = mul(sub(TV, VC), invi);
        const FV lm = mul(add(TV, VC), invi);
        // Lane j holds i = 1 + j + 8r: C - T_i is key M - i (rows M - 8 - 8r ..
        // M - 1 - 8r, lanes reversed), C + T_i key M + i (rows M + 1 + 8r ..
        // M + 8 + 8r; the last block's lane 7, C + T_M, starts the next group
        // and lands in the slack past key 2M - 1).
        store_words(sub_loose(sqr(lm), sum), s->words, M - 8 - 8 * r, true);  // to_words carries
        store_words(sub_loose(sqr(lp), sum), s->words, M + 1 + 8 * r, false);
    }
    // T_0 = J: the centre's own key, and the next centre C + J.
    uint8_t centre[32];
    to_bytes(centre, uc);
    for (int j = 0; j < 8; j++) memcpy(&s->words[j][M], centre + 4 * j, 4);
    const F lp = ::mul(::sub(t.v0, vc), inv_d0);
    const F up = ::sub(::sqr(lp), ::add(s0, t.u0));
    vc = ::sub(::mul(lp, ::sub(uc, up)), vc);
    uc = up;
}

#undef LXCPU_IFMA

inline bool available() {
    static const bool yes = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512ifma");
    return yes;
}

}  // namespace ifma

// The walk on the IFMA lanes: the same keys as Walk in the same order, in
// groups of 2048.
struct WalkIfma {
    static constexpr int SIZE = 2 * ifma::M;
    F uc, vc;
    uint64_t next = 0;
    std::unique_ptr<ifma::Scratch> s{new (std::nothrow) ifma::Scratch};  // about 170 KB

    int init(const uint8_t k[32]) {
        if (!s) return LXMFV_ERR_NOMEM;  // an error code, never an exception
        F pu, pv;
        if (int rc = start_point(k, pu, pv)) return rc;
        const ifma::Table& t = ifma::table();
        add_affine(pu, pv, t.uM, t.vM, uc, vc);
        next = 0;
        return LXMFV_OK;
    }

    // The next group; *first: the walk index of its first key.
    void advance(uint64_t* first) {
        ifma::group(uc, vc, s.get());
        *first = next;
        next += SIZE;
    }

    // The group's keys as 32-byte rows in walk order.
    const uint8_t (*keys())[32] {
        for (int k = 0; k < SIZE; k++)
            for (int j = 0; j < 8; j++) memcpy(s->buf[k] + 4 * j, &s->words[j][k], 4);
        return s->buf;
    }

    // Bit m set where key i + m of the group matches (i a multiple of 16).
    uint32_t match16(int i, const cpu_sha::Shared16& shared, const uint32_t want[4], const uint32_t mask[4]) const {
        return cpu_sha::x16::match16_shared_words(&s->words[0][i], ifma::STRIDE, shared, want, mask);
    }
};
#endif

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

// One walker: search (main.rs:292-323) from scalar `start` with Ed25519 seed
// `ed_seed`, walking with W (Walk, or WalkIfma on the IFMA lanes).
template <Hasher H, class W>
void walker(Shared* s, const uint8_t* start, const uint8_t* ed_seed) {
    uint8_t ed_pub[32];
    W w;
    if (lxmfv_ed25519_public(ed_seed, ed_pub) != LXMFV_OK || w.init(start) != LXMFV_OK) {
        s->error.store(LXMFV_ERR_STATE);
        return;
    }
    constexpr int SIZE = W::SIZE;
    static_assert(SIZE % 16 == 0, "keys are hashed 16 at a time");
    uint8_t pk[2][64], blocks[2][64], h[2][16];
    for (int j = 0; j < 2; j++) {
        memcpy(pk[j] + 32, ed_pub, 32);
        cpu_sha::address_block(s->nh, blocks[j]);
    }
    uint32_t want[4], mask[4];
    lxmfv_prefix_words(s->prefix, s->nibbles, want, mask);
    cpu_sha::Shared16 shared;
    cpu_sha::shared16_init(ed_pub, s->nh, &shared);
    while (!stopped(*s)) {
        uint64_t first;
        w.advance(&first);
        const uint8_t(*keys)[32] = H == HASH_X16 ? nullptr : w.keys();
        uint32_t hits16 = 0;
        for (int i = 0; i < SIZE; i++) {
            // Keys are hashed sixteen at a time (AVX-512: a bit per matching
            // key) or in pairs (two SHA-256 streams interleaved where the CPU
            // has the SHA extensions), and checked in walk order.
            if (H == HASH_X16) {
                if ((i & 15) == 0) hits16 = w.match16(i, shared, want, mask);
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
        s->tries.fetch_add(SIZE, std::memory_order_relaxed);
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

bool use_ifma() {
#if defined(__x86_64__)
    return ifma::available();
#else
    return false;
#endif
}

// The walk: the IFMA lanes where the CPU has them; LXMFV_CPU_WALK=scalar|ifma
// picks one (tests run each).  -1 where the choice is unknown or unavailable.
int walk_kind() {
    const char* force = getenv("LXMFV_CPU_WALK");
    if (!force) return use_ifma() ? 1 : 0;
    if (!strcmp(force, "scalar")) return 0;
    if (!strcmp(force, "ifma") && use_ifma()) return 1;
    return -1;
}

template <class W>
int walk_keys(const uint8_t start[32], uint64_t count, uint8_t* keys) {
    W w;
    if (w.init(start) != LXMFV_OK) return LXMFV_ERR_STATE;
    for (uint64_t done = 0; done < count;) {
        uint64_t first;
        w.advance(&first);
        const uint8_t(*g)[32] = w.keys();
        const uint64_t len = std::min<uint64_t>(W::SIZE, count - done);
        memcpy(keys + 32 * done, g, 32 * (size_t)len);
        done += len;
    }
    return LXMFV_OK;
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
        // Sixteen keys with one ed_pub (a walker's keys) take the path that
        // folds ed_pub and the name hash in once; others the general one.
        uint64_t i = 0;
        cpu_sha::Shared16 shared;
        const uint8_t* shared_ed = nullptr;
        for (; i + 16 <= count; i += 16) {
            const uint8_t* ed = pks + 64 * i + 32;
            bool same = true;
            for (int m = 1; m < 16 && same; m++) same = !memcmp(ed, ed + 64 * m, 32);
            if (!same) {
                cpu_sha::x16::address16_bytes(pks + 64 * i, 64, ed, 64, name_hash, out + 16 * i);
                continue;
            }
            if (!shared_ed || memcmp(shared_ed, ed, 32)) {
                cpu_sha::shared16_init(ed, name_hash, &shared);
                shared_ed = ed;
            }
            cpu_sha::x16::address16_shared_bytes(pks + 64 * i, 64, shared, out + 16 * i);
        }
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
    switch (walk_kind()) {
        case 0:
            return walk_keys<Walk>(start, count, keys);
#if defined(__x86_64__)
        case 1:
            return walk_keys<WalkIfma>(start, count, keys);
#endif
        default:
            return LXMFV_ERR_STATE;
    }
}

static int cpu_search_body(const uint8_t prefix[16], int nibbles, const uint8_t name_hash[10], int threads,
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
    // The fastest walk and hasher this CPU has; LXMFV_CPU_WALK=scalar|ifma and
    // LXMFV_CPU_HASH=c|ni|x16 pick one (tests run each), LXMFV_ERR_STATE where
    // the CPU lacks it.
    int hash = use_x16() ? HASH_X16 : use_sha_ni() ? HASH_NI : HASH_C;
    if (const char* force = getenv("LXMFV_CPU_HASH")) {
        if (!strcmp(force, "c"))
            hash = HASH_C;
        else if (!strcmp(force, "ni") && use_sha_ni())
            hash = HASH_NI;
        else if (!strcmp(force, "x16") && use_x16())
            hash = HASH_X16;
        else
            return LXMFV_ERR_STATE;
    }
    const int walk = walk_kind();
    if (walk < 0) return LXMFV_ERR_STATE;
    void (*run)(Shared*, const uint8_t*, const uint8_t*) = nullptr;
#if defined(__x86_64__)
    if (walk == 1)
        run = hash == HASH_X16 ? walker<HASH_X16, WalkIfma>
              : hash == HASH_NI ? walker<HASH_NI, WalkIfma>
                                : walker<HASH_C, WalkIfma>;
#endif
    if (!run)
        run = hash == HASH_X16 ? walker<HASH_X16, Walk> : hash == HASH_NI ? walker<HASH_NI, Walk> : walker<HASH_C, Walk>;
    for (int t = 0; t < threads; t++) {
        try {
            pool.emplace_back(run, &s, &starts[32 * (size_t)t], &eds[32 * (size_t)t]);
        } catch (...) {
            // No more threads (a process limit, or memory): the ones started
            // see the error, stop, and are joined below.
            s.error.store(LXMFV_ERR_NOMEM);
            break;
        }
    }
    while (!stopped(s)) {
        if (tries) __atomic_store_n(tries, s.tries.load(std::memory_order_relaxed), __ATOMIC_RELAXED);
        std::this_thread::sleep_for(std::chrono::milliseconds(10));
    }
    for (auto& th : pool) th.join();
    if (tries) __atomic_store_n(tries, s.tries.load(), __ATOMIC_RELAXED);
    if (s.error.load()) return s.error.load();
    return s.found.load() ? LXMFV_OK : LXMFV_STOPPED;
}

// No exception crosses the C ABI: an allocation failure before any thread
// starts becomes LXMFV_ERR_NOMEM (thread creation is handled in the body).
extern "C" int lxmfv_cpu_search(const uint8_t prefix[16], int nibbles, const uint8_t name_hash[10], int threads,
                                const uint64_t* seed, uint64_t first_walker, const int* stop, uint64_t* tries,
                                uint8_t identity[64]) {
    try {
        return cpu_search_body(prefix, nibbles, name_hash, threads, seed, first_walker, stop, tries, identity);
    } catch (const std::bad_alloc&) {
        return LXMFV_ERR_NOMEM;
    } catch (...) {
        return LXMFV_ERR_STATE;
    }
}
