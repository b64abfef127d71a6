// lxmf-vanity: the reference's command line (src/main.rs:325-499) over the
// B200 library.
//
//   lxmf-vanity <hex prefix>              search on every CPU core; writes <prefix>.identity
//   lxmf-vanity --gpu <hex prefix>        search on the GPU(s)
//   lxmf-vanity --gpu --cpu <hex prefix>  the GPU(s) and the remaining CPU cores together
//   lxmf-vanity --gpu-self-test           check the GPU against the CPU
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
// --threads (CPU threads), --walk / --batch / --lanes (kernel choice).
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
    "options:\n"
    "  --aspect NAME      destination aspect (default lxmf.delivery)\n"
    "  --devices LIST     GPUs to search on, e.g. 0,1,2,3 (default 0); first hit wins\n"
    "  --threads N        CPU threads (default: every core; with --gpu, every core but one)\n"
    "  --seed N           seeded walkers and identity (ChaCha20 stream of N) instead of OS randomness;\n"
    "                     GPU d uses seed N + d, the CPU threads seed N + (number of GPUs)\n"
    "  --walk group|xadd  the walk (default group; xadd is the x-only differential walk)\n"
    "  --batch N          keys per inversion (default 64)\n"
    "  --lanes N          walker lanes per GPU (default: one full wave)";

using Clock = std::chrono::steady_clock;

struct Options {
    bool gpu = false, cpu = false, self_test = false;
    std::string prefix_text;
    std::string aspect = "lxmf.delivery";
    std::vector<int> devices{0};
    bool seeded = false;
    uint64_t seed = 0;
    uint32_t walk = LXMFV_WALK_GROUP, batch = 64, lanes = 0;
    int threads = 0;  // CPU threads; 0: the mode's default
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

    std::string open(const Options& o, int device) {
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
            // Device d searches with the identity and walkers of seed + d.
            const uint64_t seed = o.seed + (uint64_t)device;
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
void run_device(const Options& o, const Prefix& p, int device, Shared& sh) {
    const auto started = Clock::now();
    GpuSearch g;
    std::string e = g.open(o, device);
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
    std::string e = g.open(o, o.devices[0]);
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
        else if (a == "--batch" && value(v) && parse_u64(v.c_str(), n) && n > 0 && n < 4096) o.batch = (uint32_t)n;
        else if (a == "--lanes" && value(v) && parse_u64(v.c_str(), n) && n > 0 && n < (1ull << 31)) o.lanes = (uint32_t)n;
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
    if (o.self_test) return self_test(o);
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
        for (int d : o.devices) threads.emplace_back(run_device, std::cref(o), std::cref(p), d, std::ref(sh));
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
