// lxmf-vanity: the reference's command line (src/main.rs:325-499) over the
// B200 library.
//
//   lxmf-vanity <hex prefix>              search on every CPU core; writes <prefix>.identity
//   lxmf-vanity --gpu <hex prefix>        search on the GPU(s)
//   lxmf-vanity --gpu --cpu <hex prefix>  the GPU(s) and the remaining CPU cores together
//   lxmf-vanity --gpu-self-test           check the GPU against the CPU
//   lxmf-vanity --gpu --batch-file FILE   many searches at once in the search pool
//
// Kept from the reference: the prefix rules (Prefix::parse, main.rs:206-216),
// refusing to overwrite an identity file (main.rs:467-471), the 64-byte file
// created new with mode 0600 (main.rs:484-493), the progress line every 10 s
// (main.rs:407-421), the "Found" / "About" lines (main.rs:495-498, also read by
// fleet.sh), launches grown towards 500 ms (mod.rs:148-174), every hit rebuilt
// and rechecked from scratch on the CPU before it is accepted (mod.rs:156-160),
// the self-test (mod.rs:178-207) and the three modes with their thread
// counts: every core; the GPU alone; the GPU and every core but one
// (main.rs:473-480).
// Added: --aspect (the destination aspect; default lxmf.delivery), --seed
// (seeded walkers and identity instead of OS randomness), --devices (one
// host thread per GPU, first hit wins: fleet.sh's mode in one process),
// --threads (CPU threads), --walk / --batch / --lanes (kernel choice),
// --batch-file (many searches in one persistent kernel, admitted as lanes free
// up, each retired on its first hit).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lxmfv.h"

namespace {

const char* USAGE =
    "usage: lxmf-vanity [--gpu [--cpu]] [options] <hex prefix>\n"
    "       lxmf-vanity --gpu-self-test [options]\n"
    "\n"
    "Finds a Reticulum identity whose LXMF address starts with the prefix and\n"
    "saves it to <prefix>.identity (readable only by you).\n"
    "\n"
    "  (no flag)          search on every CPU core\n"
    "  --gpu              search on the GPU (NVIDIA B200)\n"
    "  --gpu --cpu        search on the GPU and the remaining CPU cores together\n"
    "  --gpu-self-test    check the GPU's results against the CPU\n"
    "  --gpu --batch-file FILE\n"
    "                     run every search of FILE (lines '<hex prefix> [aspect]') together on\n"
    "                     one GPU; each hit is saved to <prefix>.identity as it comes in\n"
    "options:\n"
    "  --aspect NAME      destination aspect (default lxmf.delivery)\n"
    "  --devices LIST     GPUs to search on, e.g. 0,1,2,3 (default 0); first hit wins\n"
    "  --threads N        CPU threads (default: every core; with --gpu, every core but one)\n"
    "  --seed N           seeded walkers and identity (ChaCha20 stream of N) instead of OS randomness;\n"
    "                     the d-th GPU listed uses seed N + d, the CPU threads seed N + (number of\n"
    "                     GPUs); with --batch-file, search i of the file uses seed N + i\n"
    "  --walk group|xadd  the walk (default group; xadd is the x-only differential walk)\n"
    "  --batch N          keys per inversion (default 1024; --walk xadd: 128; with --batch-file, keys per\n"
    "                     group: 1024)\n"
    "  --lanes N          walker lanes per GPU (default: one full wave)";

using Clock = std::chrono::steady_clock;

struct Options {
    bool gpu = false, cpu = false, self_test = false;
    std::string prefix_text;
    std::string aspect = "lxmf.delivery";
    std::vector<int> devices{0};
    bool seeded = false;
    uint64_t seed = 0;
    uint32_t walk = LXMFV_WALK_GROUP, batch = 0, lanes = 0;  // batch 0: the library's fastest
    bool batch_given = false;
    int threads = 0;  // CPU threads; 0: the mode's default
    std::string batch_file;
};

struct Prefix {
    uint8_t bytes[16];
    int nibbles = 0;
};

std::string hex(const uint8_t* b, size_t n) {
    static const char* d = "0123456789abcdef";
    std::string s;
    for (size_t i = 0; i < n; i++) {
        s += d[b[i] >> 4];
        s += d[b[i] & 15];
    }
    return s;
}

void be_words(const uint8_t* b, size_t nwords, uint32_t* w) {
    for (size_t i = 0; i < nwords; i++)
        w[i] = (uint32_t)b[4 * i] << 24 | (uint32_t)b[4 * i + 1] << 16 | (uint32_t)b[4 * i + 2] << 8 | b[4 * i + 3];
}

// One GPU's search: its handle, lanes' start scalars and Ed25519 seed
// (GpuSearch, mod.rs:86-118).
struct GpuSearch {
    lxmfv_handle* h = nullptr;
    std::vector<uint8_t> starts;  // 32 bytes per lane
    uint8_t ed_seed[32], ed_pub[32], name_hash[10];
    uint32_t lanes = 0;
    uint64_t batch = 0;
    std::string desc;

    ~GpuSearch() { lxmfv_close(h); }

    // `index`: the device's position in --devices, which picks its seed.
    std::string open(const Options& o, int device, size_t index) {
        lxmfv_options opts{};
        opts.device = device;
        opts.lanes = o.lanes;
        opts.batch = o.batch;
        opts.walk = o.walk;
        int rc = lxmfv_open(&opts, &h);
        if (rc != LXMFV_OK) return h ? lxmfv_last_error(h) : "out of memory";
        lanes = lxmfv_threads(h);
        batch = lxmfv_batch(h);
        char buf[256];
        lxmfv_describe(h, buf, sizeof buf);
        desc = buf;
        starts.resize((size_t)lanes * 32);
        if (o.seeded) {
            // The d-th device listed searches with the identity and walkers of seed + d.
            const uint64_t seed = o.seed + (uint64_t)index;
            uint8_t ident[64];
            const uint64_t off = lxmfv_seeded_identity(seed, ident);
            memcpy(starts.data(), ident, 32);
            memcpy(ed_seed, ident + 32, 32);
            if (lanes > 1) lxmfv_seeded_scalars(seed, off, starts.data() + 32, lanes - 1);
        } else {
            // random_start_scalar per lane (main.rs:157-171) and a random Ed25519 seed (mod.rs:103).
            for (uint32_t t = 0; t < lanes; t++) {
                uint8_t* k = starts.data() + 32 * (size_t)t;
                do {
                    if (lxmfv_os_random(k, 32) != LXMFV_OK) return "no system randomness";
                } while (!lxmfv_clamp_start(k));
            }
            if (lxmfv_os_random(ed_seed, 32) != LXMFV_OK) return "no system randomness";
        }
        if (lxmfv_ed25519_public(ed_seed, ed_pub) != LXMFV_OK) return "Ed25519 key derivation failed";
        lxmfv_name_hash(o.aspect.c_str(), name_hash);
        rc = lxmfv_init_from_scalars(h, starts.data(), starts.size());
        if (rc != LXMFV_OK) return lxmfv_last_error(h);
        return "";
    }

    lxmfv_launch_args args(const Prefix& p, uint32_t iters, uint32_t dump_threads) const {
        lxmfv_launch_args a{};
        a.iters = iters;
        be_words(ed_pub, 8, a.ed);
        a.name_hash[0] = (uint32_t)name_hash[0] << 24 | (uint32_t)name_hash[1] << 16 | (uint32_t)name_hash[2] << 8 | name_hash[3];
        a.name_hash[1] = (uint32_t)name_hash[4] << 24 | (uint32_t)name_hash[5] << 16 | (uint32_t)name_hash[6] << 8 | name_hash[7];
        a.name_hash[2] = (uint32_t)name_hash[8] << 24 | (uint32_t)name_hash[9] << 16;
        lxmfv_prefix_words(p.bytes, p.nibbles, a.want, a.mask);
        // u(8B), the walk's step point, as little-endian words.
        static const uint32_t U8B[8] = {0x48c99968u, 0xf1716fedu, 0xad74a91eu, 0x7a78edcau,
                                        0xc8b65ca1u, 0xd83b884du, 0xaad65c2du, 0x275fa6d7u};
        memcpy(a.q, U8B, sizeof U8B);
        a.max_hits = 4096;
        a.dump_threads = dump_threads;
        return a;
    }

    // The identity for lane t's key number n (mod.rs:139-144).
    void identity(uint32_t t, uint64_t n, uint8_t out[64]) const {
        lxmfv_step_scalar(starts.data() + 32 * (size_t)t, n, out);
        memcpy(out + 32, ed_seed, 32);
    }
};

struct Shared {
    std::atomic<bool> found{false};
    std::atomic<uint64_t> tries{0};
    uint64_t cpu_tries = 0;  // written by lxmfv_cpu_search, read atomically
    int cpu_stop = 0;        // read by lxmfv_cpu_search, written atomically
    std::mutex mu;
    bool have_hit = false;
    uint8_t hit[64];
    std::string error;
};

// GpuSearch::run (mod.rs:148-174) on one device.
void run_device(const Options& o, const Prefix& p, int device, size_t index, Shared& sh) {
    const auto started = Clock::now();
    GpuSearch g;
    std::string e = g.open(o, device, index);
    if (!e.empty()) {
        std::lock_guard<std::mutex> l(sh.mu);
        if (sh.error.empty()) sh.error = "GPU " + std::to_string(device) + " unavailable: " + e;
        sh.found = true;
        return;
    }
    printf("%s: %u GPU threads, ready in %.1f s.\n", g.desc.c_str(), g.lanes,
           std::chrono::duration<double>(Clock::now() - started).count());
    fflush(stdout);
    const uint64_t per_iter = (uint64_t)g.lanes * g.batch;
    uint32_t iters = 1;
    std::vector<lxmfv_hit> hits(4096);
    while (!sh.found.load()) {
        const auto t0 = Clock::now();
        const lxmfv_launch_args a = g.args(p, iters, 0);
        uint32_t n = 0;
        if (lxmfv_launch(g.h, &a, hits.data(), (uint32_t)hits.size(), &n, nullptr, nullptr) != LXMFV_OK) {
            std::lock_guard<std::mutex> l(sh.mu);
            if (sh.error.empty()) sh.error = std::string("GPU: ") + lxmfv_last_error(g.h);
            sh.found = true;
            return;
        }
        const double took = std::chrono::duration<double>(Clock::now() - t0).count();
        sh.tries += per_iter * iters;
        if (n > 0) {
            // The hit with the smallest (n, lane): every lane advances in step, so
            // this is the same hit whatever the launch lengths (reproducible runs).
            const uint32_t got = n < hits.size() ? n : (uint32_t)hits.size();
            lxmfv_hit best = hits[0];
            for (uint32_t i = 1; i < got; i++)
                if (hits[i].n < best.n || (hits[i].n == best.n && hits[i].thread < best.thread)) best = hits[i];
            uint8_t ident[64], addr[16];
            g.identity(best.thread, best.n, ident);
            if (lxmfv_address_of_identity(ident, g.name_hash, addr) != LXMFV_OK ||
                !lxmfv_prefix_matches(p.bytes, p.nibbles, addr)) {
                std::lock_guard<std::mutex> l(sh.mu);
                if (sh.error.empty())
                    sh.error = "GPU hit (thread " + std::to_string(best.thread) + ", key " +
                               std::to_string(best.n) + ") failed its CPU recheck: a kernel bug";
                sh.found = true;
                return;
            }
            std::lock_guard<std::mutex> l(sh.mu);
            if (!sh.have_hit) {
                memcpy(sh.hit, ident, 64);
                sh.have_hit = true;
            }
            sh.found = true;
            return;
        }
        // Grow launches towards about 500 ms.
        if (took < 0.25 && iters < (1u << 16)) iters *= 2;
    }
}

// The CPU half: search (main.rs:292-323) on `threads` threads until a hit here
// or elsewhere.
void run_cpu(const Options& o, const Prefix& p, int threads, Shared& sh) {
    uint8_t nh[10], ident[64];
    lxmfv_name_hash(o.aspect.c_str(), nh);
    const uint64_t seed = o.seed + (o.gpu ? (uint64_t)o.devices.size() : 0);
    const int rc = lxmfv_cpu_search(p.bytes, p.nibbles, nh, threads, o.seeded ? &seed : nullptr, 0, &sh.cpu_stop,
                                    &sh.cpu_tries, ident);
    if (rc == LXMFV_STOPPED) return;
    std::lock_guard<std::mutex> l(sh.mu);
    if (rc == LXMFV_OK) {
        if (!sh.have_hit) {
            memcpy(sh.hit, ident, 64);
            sh.have_hit = true;
        }
    } else if (sh.error.empty()) {
        sh.error = rc == LXMFV_ERR_RECHECK ? "internal error: a CPU hit failed its recheck; not saving it"
                                           : "CPU search failed (code " + std::to_string(rc) + ")";
    }
    sh.found = true;
}

int self_test(const Options& o) {
    GpuSearch g;
    const auto started = Clock::now();
    std::string e = g.open(o, o.devices[0], 0);
    if (!e.empty()) {
        fprintf(stderr, "GPU unavailable: %s\n", e.c_str());
        return 1;
    }
    printf("%s: %u GPU threads, ready in %.1f s.\n", g.desc.c_str(), g.lanes,
           std::chrono::duration<double>(Clock::now() - started).count());
    const uint32_t dump_threads = g.lanes < 256 ? g.lanes : 256;
    Prefix any;
    any.nibbles = lxmfv_prefix_parse("b0", any.bytes);  // about 1 key in 256
    const lxmfv_launch_args a = g.args(any, 1, dump_threads);
    std::vector<lxmfv_hit> hits(4096);
    std::vector<uint32_t> dump((size_t)dump_threads * g.batch * 8);
    uint32_t n = 0;
    if (lxmfv_launch(g.h, &a, hits.data(), (uint32_t)hits.size(), &n, dump.data(), nullptr) != LXMFV_OK) {
        fprintf(stderr, "Self-test FAILED: %s\n", lxmfv_last_error(g.h));
        return 2;
    }
    for (uint32_t t = 0; t < dump_threads; t++) {
        for (uint64_t i = 0; i < g.batch; i++) {
            uint8_t k[32], expected[32];
            lxmfv_step_scalar(g.starts.data() + 32 * (size_t)t, i, k);
            lxmfv_x25519_base(k, expected);
            if (memcmp(expected, &dump[((size_t)t * g.batch + i) * 8], 32) != 0) {
                fprintf(stderr, "Self-test FAILED: public key mismatch: thread %u, key %llu\n", t, (unsigned long long)i);
                return 2;
            }
        }
    }
    const uint32_t got = n < hits.size() ? n : (uint32_t)hits.size();
    if (got < 100) {
        fprintf(stderr, "Self-test FAILED: only %u hits for a 2-digit prefix; expected thousands\n", got);
        return 2;
    }
    for (uint32_t i = 0; i < got; i++) {
        uint8_t ident[64], addr[16];
        g.identity(hits[i].thread, hits[i].n, ident);
        if (lxmfv_address_of_identity(ident, g.name_hash, addr) != LXMFV_OK ||
            !lxmfv_prefix_matches(any.bytes, any.nibbles, addr)) {
            fprintf(stderr, "Self-test FAILED: hit (thread %u, key %llu) failed its CPU recheck\n", hits[i].thread,
                    (unsigned long long)hits[i].n);
            return 2;
        }
    }
    printf("Self-test passed: %llu public keys match X25519, %u hits for 'b0' all recheck on the CPU.\n",
           (unsigned long long)dump_threads * g.batch, got);
    return 0;
}

// ---- --batch-file: many searches in the search pool. ----

struct BatchSearch {
    std::string text, aspect, path;
    Prefix p;
    uint8_t nh[10], ed_seed[32], ed_pub[32];
    std::vector<uint8_t> starts;  // 32 bytes per lane
    uint32_t lanes = 0, id = 0;
    bool active = false, done = false;
};

// Lanes for a search of `nibbles` digits: 64 for 5 or fewer, 16 times more per
// further digit (so expected steps to a hit stay about level), at most 2^17.
// A function of the search alone, so that its hit does not depend on the mix.
uint32_t batch_lanes(int nibbles) {
    double l = 64.0 * std::pow(16.0, std::max(0, nibbles - 5));
    return (uint32_t)std::min(131072.0, l);
}

bool read_batch_file(const Options& o, std::vector<BatchSearch>& out) {
    FILE* f = fopen(o.batch_file.c_str(), "r");
    if (!f) {
        fprintf(stderr, "could not read %s: %s\n", o.batch_file.c_str(), strerror(errno));
        return false;
    }
    char line[1024];
    int lineno = 0;
    bool ok = true;
    while (ok && fgets(line, sizeof line, f)) {
        lineno++;
        char* hash = strchr(line, '#');
        if (hash) *hash = 0;
        char pfx[256] = {0}, asp[512] = {0}, extra[8] = {0};
        const int n = sscanf(line, "%255s %511s %7s", pfx, asp, extra);
        if (n <= 0) continue;
        if (n > 2) {
            fprintf(stderr, "%s:%d: expected '<hex prefix> [aspect]'\n", o.batch_file.c_str(), lineno);
            ok = false;
            break;
        }
        BatchSearch b;
        b.text = pfx;
        for (auto& c : b.text) c = (char)tolower((unsigned char)c);
        b.aspect = n == 2 ? asp : o.aspect;
        b.p.nibbles = lxmfv_prefix_parse(b.text.c_str(), b.p.bytes);
        if (b.p.nibbles < 0) {
            fprintf(stderr, "%s:%d: '%s' isn't 1 to 32 hex digits: use 0-9 and a-f only (zero, not the letter O).\n",
                    o.batch_file.c_str(), lineno, pfx);
            ok = false;
            break;
        }
        b.path = b.text + ".identity";
        struct stat st;
        if (stat(b.path.c_str(), &st) == 0) {
            fprintf(stderr, "%s already exists; not overwriting it.\n", b.path.c_str());
            ok = false;
            break;
        }
        for (const auto& prev : out)
            if (prev.text == b.text) {
                fprintf(stderr, "%s:%d: prefix %s is listed twice (both would write %s)\n", o.batch_file.c_str(),
                        lineno, b.text.c_str(), b.path.c_str());
                ok = false;
            }
        out.push_back(std::move(b));
    }
    fclose(f);
    if (ok && out.empty()) {
        fprintf(stderr, "%s lists no searches\n", o.batch_file.c_str());
        ok = false;
    }
    return ok;
}

// Start scalars and identity of search i: seeded (seed + i) or from the OS.
std::string prepare_batch_search(const Options& o, size_t i, BatchSearch& b) {
    b.lanes = o.lanes ? (o.lanes + 31) / 32 * 32 : batch_lanes(b.p.nibbles);
    b.starts.resize((size_t)b.lanes * 32);
    if (o.seeded) {
        uint8_t ident[64];
        const uint64_t off = lxmfv_seeded_identity(o.seed + i, ident);
        memcpy(b.starts.data(), ident, 32);
        memcpy(b.ed_seed, ident + 32, 32);
        if (b.lanes > 1) lxmfv_seeded_scalars(o.seed + i, off, b.starts.data() + 32, b.lanes - 1);
    } else {
        for (uint32_t t = 0; t < b.lanes; t++) {
            uint8_t* k = b.starts.data() + 32 * (size_t)t;
            do {
                if (lxmfv_os_random(k, 32) != LXMFV_OK) return "no system randomness";
            } while (!lxmfv_clamp_start(k));
        }
        if (lxmfv_os_random(b.ed_seed, 32) != LXMFV_OK) return "no system randomness";
    }
    if (lxmfv_ed25519_public(b.ed_seed, b.ed_pub) != LXMFV_OK) return "Ed25519 key derivation failed";
    lxmfv_name_hash(b.aspect.c_str(), b.nh);
    return "";
}

lxmfv_search_desc batch_desc(const BatchSearch& b) {
    lxmfv_search_desc d{};
    be_words(b.ed_pub, 8, d.ed);
    d.name_hash[0] = (uint32_t)b.nh[0] << 24 | (uint32_t)b.nh[1] << 16 | (uint32_t)b.nh[2] << 8 | b.nh[3];
    d.name_hash[1] = (uint32_t)b.nh[4] << 24 | (uint32_t)b.nh[5] << 16 | (uint32_t)b.nh[6] << 8 | b.nh[7];
    d.name_hash[2] = (uint32_t)b.nh[8] << 24 | (uint32_t)b.nh[9] << 16;
    lxmfv_prefix_words(b.p.bytes, b.p.nibbles, d.want, d.mask);
    d.lanes = b.lanes;
    return d;
}

bool write_identity(const std::string& path, const uint8_t ident[64]) {
    // The file holds a private key: created new, readable only by the owner.
    const int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_EXCL, 0600);
    if (fd < 0) {
        fprintf(stderr, "could not create %s: %s\n", path.c_str(), strerror(errno));
        return false;
    }
    const bool ok = write(fd, ident, 64) == 64;
    return close(fd) == 0 && ok;
}

int run_batch_file(const Options& o) {
    std::vector<BatchSearch> searches;
    if (!read_batch_file(o, searches)) return 1;
    const auto start = Clock::now();
    lxmfv_pool_options po{};
    po.device = o.devices[0];
    po.batch = o.batch_given ? o.batch : 0;  // 0: the pool's default group of 1024 keys
    po.max_searches = (uint32_t)std::min<size_t>(4096, searches.size());
    lxmfv_pool* pool = nullptr;
    int rc = lxmfv_pool_open(&po, &pool);
    lxmfv_pool_info_t info{};
    if (rc == LXMFV_OK) rc = lxmfv_pool_info(pool, &info);
    if (rc != LXMFV_OK) {
        fprintf(stderr, "GPU unavailable: %s\n", pool ? lxmfv_pool_last_error(pool) : "out of memory");
        lxmfv_pool_close(pool);
        return 2;
    }
    for (size_t i = 0; i < searches.size(); i++) {
        const std::string e = prepare_batch_search(o, i, searches[i]);
        if (!e.empty()) {
            fprintf(stderr, "%s\n", e.c_str());
            lxmfv_pool_close(pool);
            return 2;
        }
        if (searches[i].lanes > info.capacity_lanes) {
            fprintf(stderr, "%s: %u lanes exceed the pool's %u\n", searches[i].text.c_str(), searches[i].lanes,
                    info.capacity_lanes);
            lxmfv_pool_close(pool);
            return 1;
        }
    }
    printf("%zu searches on the GPU pool (%u lanes, %u keys per group), ready in %.1f s.\n", searches.size(),
           info.capacity_lanes, info.batch, std::chrono::duration<double>(Clock::now() - start).count());
    fflush(stdout);

    std::vector<lxmfv_pool_hit> hits(65536);
    std::vector<int> by_id(po.max_searches, -1);
    size_t next = 0, found = 0;
    uint64_t tries = 0;
    uint32_t groups = 1;
    int status = 0;
    auto next_report = Clock::now() + std::chrono::seconds(10);
    while (found < searches.size() && status == 0) {
        // Admit waiting searches, in file order, while lanes and slots are free.
        while (next < searches.size()) {
            BatchSearch& b = searches[next];
            const lxmfv_search_desc d = batch_desc(b);
            rc = lxmfv_pool_submit(pool, &d, b.starts.data(), &b.id);
            if (rc == LXMFV_ERR_OVERFLOW) break;
            if (rc != LXMFV_OK) {
                fprintf(stderr, "GPU: %s\n", lxmfv_pool_last_error(pool));
                status = 2;
                break;
            }
            b.active = true;
            by_id[b.id] = (int)next;
            next++;
        }
        if (status) break;
        uint64_t active_lanes = 0;
        for (const auto& b : searches) active_lanes += b.active ? b.lanes : 0;
        uint32_t n = 0;
        if (lxmfv_pool_step(pool, groups) != LXMFV_OK ||
            lxmfv_pool_poll(pool, hits.data(), (uint32_t)hits.size(), &n) != LXMFV_OK) {
            fprintf(stderr, "GPU: %s\n", lxmfv_pool_last_error(pool));
            status = 2;
            break;
        }
        if (n > hits.size()) {
            fprintf(stderr, "GPU: %u hits in one step exceed the %zu held; use longer prefixes\n", n, hits.size());
            status = 2;
            break;
        }
        tries += active_lanes * info.batch * groups;
        // Per search, the hit with the smallest (n, lane): the first in walk order.
        std::vector<const lxmfv_pool_hit*> first(po.max_searches, nullptr);
        for (uint32_t i = 0; i < n; i++) {
            const lxmfv_pool_hit& h = hits[i];
            if (h.search >= by_id.size() || by_id[h.search] < 0) continue;
            const lxmfv_pool_hit*& f = first[h.search];
            if (!f || h.n < f->n || (h.n == f->n && h.lane < f->lane)) f = &h;
        }
        for (uint32_t id = 0; id < first.size() && status == 0; id++) {
            if (!first[id]) continue;
            BatchSearch& b = searches[(size_t)by_id[id]];
            uint8_t ident[64], addr[16];
            lxmfv_step_scalar(b.starts.data() + 32 * (size_t)first[id]->lane, first[id]->n, ident);
            memcpy(ident + 32, b.ed_seed, 32);
            if (lxmfv_address_of_identity(ident, b.nh, addr) != LXMFV_OK ||
                !lxmfv_prefix_matches(b.p.bytes, b.p.nibbles, addr)) {
                fprintf(stderr, "GPU hit for %s (lane %u, key %llu) failed its CPU recheck: a kernel bug\n",
                        b.text.c_str(), first[id]->lane, (unsigned long long)first[id]->n);
                status = 2;
                break;
            }
            if (!write_identity(b.path, ident)) {
                status = 1;
                break;
            }
            lxmfv_pool_retire(pool, id);
            by_id[id] = -1;
            b.active = false;
            b.done = true;
            found++;
            const uint64_t own = first[id]->n * b.lanes + first[id]->lane + 1;
            printf("Found %s (%s) after about %llu tries. Saved to %s\n", hex(addr, 16).c_str(), b.aspect.c_str(),
                   (unsigned long long)own, b.path.c_str());
            fflush(stdout);
        }
        // Grow steps towards about 100 ms of GPU time.
        if (lxmfv_pool_last_step_ms(pool) < 50.0f && groups < 64) groups *= 2;
        if (Clock::now() >= next_report) {
            const double el = std::chrono::duration<double>(Clock::now() - start).count();
            printf("%zu of %zu found; %.0f tries, %.0f/s\n", found, searches.size(), (double)tries, tries / el);
            fflush(stdout);
            next_report += std::chrono::seconds(10);
        }
    }
    lxmfv_pool_close(pool);
    if (status) return status;
    const double elapsed = std::chrono::duration<double>(Clock::now() - start).count();
    printf("All %zu found: about %llu tries in %.1f s (%.0f/s).\n", searches.size(), (unsigned long long)tries,
           elapsed, (double)tries / elapsed);
    return 0;
}

bool parse_devices(const std::string& s, std::vector<int>& out) {
    out.clear();
    size_t i = 0;
    while (i < s.size()) {
        size_t j = s.find(',', i);
        if (j == std::string::npos) j = s.size();
        const std::string part = s.substr(i, j - i);
        if (part.empty() || part.find_first_not_of("0123456789") != std::string::npos) return false;
        out.push_back(atoi(part.c_str()));
        i = j + 1;
    }
    return !out.empty();
}

bool parse_u64(const char* s, uint64_t& v) {
    char* end = nullptr;
    errno = 0;
    v = strtoull(s, &end, 0);
    return errno == 0 && end && *end == 0 && *s;
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    std::vector<std::string> words;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto value = [&](std::string& out) {
            if (i + 1 >= argc) return false;
            out = argv[++i];
            return true;
        };
        std::string v;
        uint64_t n = 0;
        if (a == "--gpu") o.gpu = true;
        else if (a == "--cpu") o.cpu = true;
        else if (a == "--gpu-self-test") o.self_test = true;
        else if (a == "--aspect" && value(v) && !v.empty()) o.aspect = v;
        else if (a == "--devices" && value(v) && parse_devices(v, o.devices)) {}
        else if (a == "--seed" && value(v) && parse_u64(v.c_str(), n)) { o.seeded = true; o.seed = n; }
        else if (a == "--walk" && value(v) && (v == "group" || v == "xadd")) o.walk = v == "group" ? LXMFV_WALK_GROUP : LXMFV_WALK_XADD;
        else if (a == "--batch" && value(v) && parse_u64(v.c_str(), n) && n > 0 && n < 4096) { o.batch = (uint32_t)n; o.batch_given = true; }
        else if (a == "--lanes" && value(v) && parse_u64(v.c_str(), n) && n > 0 && n < (1ull << 31)) o.lanes = (uint32_t)n;
        else if (a == "--batch-file" && value(v) && !v.empty()) o.batch_file = v;
        else if (a == "--threads" && value(v) && parse_u64(v.c_str(), n) && n > 0 && n <= LXMFV_CPU_MAX_THREADS) o.threads = (int)n;
        else if (a.rfind("--", 0) == 0) {
            fprintf(stderr, "%s\n", USAGE);
            return 1;
        } else words.push_back(a);
    }
    if (o.cpu && !o.gpu) {
        fprintf(stderr, "%s\n", USAGE);
        return 1;
    }
    // The fastest keys per inversion of each walk (the x-only walk builds at most 128).
    if (!o.batch_given && o.walk == LXMFV_WALK_XADD) o.batch = 128;
    if (o.self_test) return self_test(o);
    if (!o.batch_file.empty()) {
        if (!o.gpu || o.cpu || !words.empty()) {
            fprintf(stderr, "%s\n", USAGE);
            return 1;
        }
        return run_batch_file(o);
    }
    if (words.size() != 1) {
        fprintf(stderr, "%s\n", USAGE);
        return 1;
    }
    Prefix p;
    std::string text = words[0];
    for (auto& c : text) c = (char)tolower((unsigned char)c);
    p.nibbles = lxmfv_prefix_parse(text.c_str(), p.bytes);
    if (p.nibbles < 0) {
        fprintf(stderr, "'%s' isn't 1 to 32 hex digits: use 0-9 and a-f only (zero, not the letter O).\n",
                text.c_str());
        return 1;
    }
    const std::string path = text + ".identity";
    struct stat st;
    if (stat(path.c_str(), &st) == 0) {
        fprintf(stderr, "%s already exists; not overwriting it.\n", path.c_str());
        return 1;
    }
    printf("Looking for an LXMF address starting %s.\n", text.c_str());
    const double expected = std::pow(16.0, p.nibbles);
    // Every core; with the GPU, one core per GPU is left to drive it (main.rs:473-480).
    const int cores = (int)std::max(1u, std::thread::hardware_concurrency());
    int cpu_threads = o.threads;
    if (!cpu_threads) cpu_threads = !o.gpu ? cores : o.cpu ? std::max(1, cores - (int)o.devices.size()) : 0;
    if (o.gpu && !o.cpu) cpu_threads = 0;
    std::string on;
    if (o.gpu) on = std::to_string(o.devices.size()) + (o.devices.size() > 1 ? " GPUs" : " GPU");
    if (cpu_threads)
        on += (on.empty() ? "" : " and ") + std::to_string(cpu_threads) + (cpu_threads > 1 ? " CPU threads" : " CPU thread");
    printf("Searching on %s; about %.0f tries on average.\n", on.c_str(), expected);
    fflush(stdout);

    Shared sh;
    const auto start = Clock::now();
    std::vector<std::thread> threads;
    if (o.gpu)
        for (size_t i = 0; i < o.devices.size(); i++)
            threads.emplace_back(run_device, std::cref(o), std::cref(p), o.devices[i], i, std::ref(sh));
    if (cpu_threads) threads.emplace_back(run_cpu, std::cref(o), std::cref(p), cpu_threads, std::ref(sh));
    auto all_tries = [&sh]() { return sh.tries.load() + __atomic_load_n(&sh.cpu_tries, __ATOMIC_RELAXED); };
    auto next_report = start + std::chrono::seconds(10);
    while (!sh.found.load()) {
        std::this_thread::sleep_for(std::chrono::milliseconds(50));
        if (Clock::now() >= next_report) {
            const double done = (double)all_tries();
            const double rate = done / std::chrono::duration<double>(Clock::now() - start).count();
            if (done < expected)
                printf("%.0f tries, %.0f/s; the average is about %.0f min away\n", done, rate,
                       (expected - done) / rate / 60.0);
            else
                printf("%.0f tries, %.0f/s; past the average, still searching\n", done, rate);
            fflush(stdout);
            next_report += std::chrono::seconds(10);
        }
    }
    __atomic_store_n(&sh.cpu_stop, 1, __ATOMIC_RELAXED);
    for (auto& t : threads) t.join();
    if (!sh.error.empty() && !sh.have_hit) {
        fprintf(stderr, "%s\n", sh.error.c_str());
        return 2;
    }
    // The file holds a private key: created new, readable only by the owner.
    const int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_EXCL, 0600);
    if (fd < 0) {
        fprintf(stderr, "could not create %s: %s\n", path.c_str(), strerror(errno));
        return 1;
    }
    if (write(fd, sh.hit, 64) != 64 || close(fd) != 0) {
        fprintf(stderr, "could not write the identity\n");
        return 1;
    }
    const double elapsed = std::chrono::duration<double>(Clock::now() - start).count();
    uint8_t addr[16], nh[10];
    lxmfv_name_hash(o.aspect.c_str(), nh);
    lxmfv_address_of_identity(sh.hit, nh, addr);
    const uint64_t tried = all_tries();
    printf("Found %s\n", hex(addr, 16).c_str());
    printf("About %llu tries in %.1f s (%.0f/s). Saved to %s\n", (unsigned long long)tried, elapsed,
           (double)tried / elapsed, path.c_str());
    return 0;
}
