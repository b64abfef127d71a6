// Host-side rules of the reference's search (CPU): prefixes, scalars, seeded
// draws, and the from-scratch recheck of a hit.
//
// The recheck uses OpenSSL's X25519, Ed25519 and SHA-256, an implementation
// independent of the GPU kernels, as the reference rechecks with
// x25519-dalek, ed25519-dalek and sha2 (address_of_identity, main.rs:191-197).
#include <openssl/evp.h>
#include <openssl/sha.h>
#include <sys/random.h>

#include <cerrno>
#include <cstring>

#include "../../include/lxmfv.h"

extern "C" {

int lxmfv_prefix_parse(const char* text, uint8_t bytes[16]) {
    if (!text || !bytes) return LXMFV_ERR_ARG;
    const size_t n = strlen(text);
    if (n == 0 || n > 32) return LXMFV_ERR_ARG;
    uint8_t b[16] = {0};
    for (size_t i = 0; i < n; i++) {
        const char c = text[i];
        int v;
        if (c >= '0' && c <= '9') v = c - '0';
        else if (c >= 'a' && c <= 'f') v = c - 'a' + 10;
        else if (c >= 'A' && c <= 'F') v = c - 'A' + 10;
        else return LXMFV_ERR_ARG;
        b[i / 2] |= (uint8_t)(v << (i % 2 == 0 ? 4 : 0));
    }
    memcpy(bytes, b, 16);
    return (int)n;
}

int lxmfv_prefix_matches(const uint8_t bytes[16], int nibbles, const uint8_t address[16]) {
    if (!bytes || !address || nibbles < 1 || nibbles > 32) return 0;
    const int whole = nibbles / 2;
    if (memcmp(address, bytes, (size_t)whole) != 0) return 0;
    return nibbles % 2 == 0 || (address[whole] >> 4) == (bytes[whole] >> 4);
}

void lxmfv_prefix_words(const uint8_t bytes[16], int nibbles, uint32_t want[4], uint32_t mask[4]) {
    uint8_t w[16] = {0}, m[16] = {0};
    for (int i = 0; i < nibbles && i < 32; i++) {
        const int shift = i % 2 == 0 ? 4 : 0;
        m[i / 2] |= (uint8_t)(0xF << shift);
        w[i / 2] |= (uint8_t)(((bytes[i / 2] >> shift) & 0xF) << shift);
    }
    for (int k = 0; k < 4; k++) {
        want[k] = (uint32_t)w[4 * k] << 24 | (uint32_t)w[4 * k + 1] << 16 | (uint32_t)w[4 * k + 2] << 8 | w[4 * k + 3];
        mask[k] = (uint32_t)m[4 * k] << 24 | (uint32_t)m[4 * k + 1] << 16 | (uint32_t)m[4 * k + 2] << 8 | m[4 * k + 3];
    }
}

void lxmfv_name_hash(const char* aspect, uint8_t out[10]) {
    uint8_t h[32];
    SHA256((const unsigned char*)aspect, strlen(aspect), h);
    memcpy(out, h, 10);
}

void lxmfv_step_scalar(const uint8_t k[32], uint64_t n, uint8_t out[32]) {
    // k + 8n with 8n up to 67 bits: a byte-wise carry chain.
    unsigned __int128 carry = (unsigned __int128)n * 8;
    for (int i = 0; i < 32; i++) {
        const unsigned __int128 sum = (unsigned __int128)k[i] + (carry & 0xFF);
        out[i] = (uint8_t)sum;
        carry = (carry >> 8) + (sum >> 8);
    }
}

void lxmfv_previous_scalar(const uint8_t k[32], uint8_t out[32]) {
    int borrow = 8;
    for (int i = 0; i < 32; i++) {
        const int v = (int)k[i] - borrow;
        out[i] = (uint8_t)(v & 0xFF);
        borrow = v < 0;
    }
}

int lxmfv_clamp_start(uint8_t k[32]) {
    k[0] &= 248;
    k[31] &= 127;
    k[31] |= 64;
    bool high_all_set = k[31] == 127, low_all_clear = k[31] == 64;
    for (int i = 9; i < 31; i++) high_all_set = high_all_set && k[i] == 0xFF;
    for (int i = 0; i < 31; i++) low_all_clear = low_all_clear && k[i] == 0;
    return !high_all_set && !low_all_clear;
}

// ---- ChaCha20 keystream (RFC 8439, section 2.3).

static inline uint32_t rotl32(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }

static void chacha_block(uint64_t seed, uint32_t counter, uint8_t out[64]) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, (uint32_t)seed, (uint32_t)(seed >> 32), 0,
                      0, 0, 0, 0, 0, counter, 0, 0, 0};
    uint32_t x[16];
    memcpy(x, s, sizeof x);
    auto qr = [&](int a, int b, int c, int d) {
        x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16);
        x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12);
        x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);
        x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
    };
    for (int i = 0; i < 10; i++) {
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
    }
    for (int i = 0; i < 16; i++) {
        const uint32_t v = x[i] + s[i];
        out[4 * i] = (uint8_t)v; out[4 * i + 1] = (uint8_t)(v >> 8);
        out[4 * i + 2] = (uint8_t)(v >> 16); out[4 * i + 3] = (uint8_t)(v >> 24);
    }
}

static void chacha_stream(uint64_t seed, uint64_t offset, uint8_t* out, size_t len) {
    uint8_t blk[64];
    while (len > 0) {
        const size_t skip = offset % 64;
        size_t take = 64 - skip;
        if (take > len) take = len;
        chacha_block(seed, (uint32_t)(offset / 64), blk);
        memcpy(out, blk + skip, take);
        out += take;
        len -= take;
        offset += take;
    }
}

uint64_t lxmfv_seeded_scalars(uint64_t seed, uint64_t offset, uint8_t* scalars, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) {
        for (;;) {
            chacha_stream(seed, offset, scalars + 32 * i, 32);
            offset += 32;
            if (lxmfv_clamp_start(scalars + 32 * i)) break;
        }
    }
    return offset;
}

uint64_t lxmfv_seeded_identity(uint64_t seed, uint8_t identity[64]) {
    uint64_t off = lxmfv_seeded_scalars(seed, 0, identity, 1);
    chacha_stream(seed, off, identity + 32, 32);
    return off + 32;
}

int lxmfv_os_random(uint8_t* out, size_t len) {
    size_t got = 0;
    while (got < len) {
        const ssize_t r = getrandom(out + got, len - got, 0);
        if (r < 0) {
            if (errno == EINTR) continue;
            return LXMFV_ERR_STATE;
        }
        got += (size_t)r;
    }
    return LXMFV_OK;
}

// ---- OpenSSL: the independent recheck.

static int raw_public(int type, const uint8_t priv[32], uint8_t out[32]) {
    EVP_PKEY* k = EVP_PKEY_new_raw_private_key(type, nullptr, priv, 32);
    if (!k) return LXMFV_ERR_STATE;
    size_t len = 32;
    const int ok = EVP_PKEY_get_raw_public_key(k, out, &len);
    EVP_PKEY_free(k);
    return (ok == 1 && len == 32) ? LXMFV_OK : LXMFV_ERR_STATE;
}

int lxmfv_ed25519_public(const uint8_t seed[32], uint8_t out[32]) { return raw_public(EVP_PKEY_ED25519, seed, out); }

int lxmfv_x25519_base(const uint8_t k[32], uint8_t out[32]) { return raw_public(EVP_PKEY_X25519, k, out); }

int lxmfv_address_of_identity(const uint8_t identity[64], const uint8_t name_hash[10], uint8_t out[16]) {
    uint8_t pk[64], ih[32], mat[26], h[32];
    if (int rc = lxmfv_x25519_base(identity, pk)) return rc;
    if (int rc = lxmfv_ed25519_public(identity + 32, pk + 32)) return rc;
    SHA256(pk, 64, ih);
    memcpy(mat, name_hash, 10);
    memcpy(mat + 10, ih, 16);
    SHA256(mat, 26, h);
    memcpy(out, h, 16);
    return LXMFV_OK;
}

}  // extern "C"
