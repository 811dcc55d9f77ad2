// ref_driver.cpp -- harness around the reference's own hot-path sources.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file against the
// UNMODIFIED "Mass Prime Siever/Math.hpp" and "Sieve.hpp" where they lie in
// the reference tree (with the two-header Boost shim in oracle/shim/), into
// oracle/_ref/libmps_ref.so and oracle/_ref/mps_ref.  It pins the C
// restatement in mps_oracle.c and is the CPU baseline ("reference" kind).
//
// The chunk loop mirrors process_chunk's CPU branch (Worker.hpp:195-303):
// segmented_sieve over the chunk, then run_bsgs per prime with an
// mt19937_64 seeded by (thread_id + 1) ^ chunk.low (Worker.hpp:247-248).
// The thread pool mirrors run_worker_pool (Worker.hpp:305-367): workers pop
// contiguous chunks of the P range from a shared cursor.
#include "Sieve.hpp"   // reference: Sieve.hpp, Math.hpp, Types.hpp, Portable.hpp

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

using namespace siever;

extern "C" {

typedef struct ref_item {
    int64_t b_hi;
    uint64_t b_lo;
    int64_t c_hi;
    uint64_t c_lo;
    uint64_t P0, P1;
    int64_t N0, N1;
    uint64_t mod, res;
} ref_item;

typedef struct ref_relation {
    uint64_t p, M, q;
} ref_relation;
}

static WorkItem to_work_item(const ref_item* it) {
    WorkItem w;
    w.b = (Int128)(((unsigned __int128)(uint64_t)it->b_hi << 64) | it->b_lo);
    w.c = (Int128)(((unsigned __int128)(uint64_t)it->c_hi << 64) | it->c_lo);
    w.P0 = (Int128)it->P0;
    w.P0_original = w.P0;
    w.P1 = (Int128)it->P1;
    w.N0 = (Int128)it->N0;
    w.N1 = (Int128)it->N1;
    w.cls_mod = it->mod == 0 ? 1 : it->mod;
    w.cls_res = it->res;
    return w;
}

static const std::vector<uint32_t>& small_primes_for(const WorkItem& w) {
    static std::mutex lock;
    static std::vector<uint32_t> cache;
    static uint64_t cache_limit = 0;
    std::lock_guard<std::mutex> g(lock);
    const uint64_t lim = sieve_limit_for(w);
    if (cache.empty() || cache_limit < lim) {
        cache = sieve_small_primes(lim);
        cache_limit = lim;
    }
    return cache;
}

static void chunk(const WorkItem& w, const std::vector<uint32_t>& sp, uint64_t lo, uint64_t hi, int thread_id,
                  std::vector<Relation>& rel, uint64_t* nprimes) {
    std::vector<uint64_t> primes;
    segmented_sieve((UInt128)lo, (UInt128)hi, sp, primes);
    if (nprimes) *nprimes += primes.size();
    std::mt19937_64 rng(static_cast<uint64_t>(thread_id + 1) ^ lo);
    for (const uint64_t p : primes) {
        Relation r;
        if (run_bsgs(p, w, r, rng)) rel.push_back(r);
    }
}

extern "C" {

int ref_is_prime64(uint64_t n) { return is_prime64(n) ? 1 : 0; }

// run_bsgs on one prime (Math.hpp:377-486); 1 if it yields a relation.
int ref_run_bsgs(uint64_t p, const ref_item* item, ref_relation* out) {
    const WorkItem w = to_work_item(item);
    std::mt19937_64 rng(1);
    Relation r;
    if (!run_bsgs(p, w, r, rng)) return 0;
    *out = ref_relation{r.p, r.M, r.q};
    return 1;
}

uint64_t ref_mult_order(uint64_t b, uint64_t p) {
    std::mt19937_64 rng(1);
    return multiplicative_order(b, p, rng);
}

size_t ref_sieve(uint64_t lo, uint64_t hi, uint64_t* out, size_t cap) {
    WorkItem w;
    w.P1 = (Int128)hi;
    const std::vector<uint32_t>& sp = small_primes_for(w);
    std::vector<uint64_t> primes;
    segmented_sieve((UInt128)lo, (UInt128)hi, sp, primes);
    for (size_t i = 0; i < primes.size() && i < cap; ++i) out[i] = primes[i];
    return primes.size();
}

// Relations of the primes in [lo, hi) (the item's P0/P1 set only the small-prime limit).
size_t ref_chunk_relations(uint64_t lo, uint64_t hi, const ref_item* item, ref_relation* out, size_t cap,
                           uint64_t* nprimes) {
    const WorkItem w = to_work_item(item);
    const std::vector<uint32_t>& sp = small_primes_for(w);
    std::vector<Relation> rel;
    if (nprimes) *nprimes = 0;
    chunk(w, sp, lo, hi, 0, rel, nprimes);
    for (size_t i = 0; i < rel.size() && i < cap; ++i) out[i] = ref_relation{rel[i].p, rel[i].M, rel[i].q};
    return rel.size();
}

// [lo, hi) split into chunks of `chunk_size` integers over `threads` workers; relations sorted by p.
size_t ref_relations_threaded(uint64_t lo, uint64_t hi, const ref_item* item, ref_relation* out, size_t cap,
                              int threads, uint64_t chunk_size, uint64_t* nprimes) {
    const WorkItem w = to_work_item(item);
    const std::vector<uint32_t>& sp = small_primes_for(w);
    if (threads < 1) threads = 1;
    if (chunk_size == 0) chunk_size = 1ULL << 24;
    std::atomic<uint64_t> cursor{lo};
    std::atomic<uint64_t> total_primes{0};
    std::mutex merge;
    std::vector<Relation> all;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        pool.emplace_back([&, t] {
            std::vector<Relation> rel;
            uint64_t np = 0;
            for (;;) {
                const uint64_t a = cursor.fetch_add(chunk_size);
                if (a >= hi) break;
                const uint64_t b = (hi - a > chunk_size) ? a + chunk_size : hi;
                chunk(w, sp, a, b, t, rel, &np);
            }
            total_primes += np;
            std::lock_guard<std::mutex> g(merge);
            all.insert(all.end(), rel.begin(), rel.end());
        });
    }
    for (std::thread& th : pool) th.join();
    std::sort(all.begin(), all.end(), [](const Relation& x, const Relation& y) { return x.p < y.p; });
    for (size_t i = 0; i < all.size() && i < cap; ++i) out[i] = ref_relation{all[i].p, all[i].M, all[i].q};
    if (nprimes) *nprimes = total_primes.load();
    return all.size();
}

}  // extern "C"

#ifdef MPS_REF_MAIN
// mps_ref b c P0 P1 N0 N1 [mod res [threads]]: relations.p lines sorted by p on stdout,
// "primes=<n> relations=<k> seconds=<s>" on stderr.
int main(int argc, char** argv) {
    if (argc < 7) {
        std::fprintf(stderr, "usage: mps_ref b c P0 P1 N0 N1 [mod res [threads]]\n");
        return 2;
    }
    ref_item it{};
    const long long b = std::atoll(argv[1]), c = std::atoll(argv[2]);
    it.b_hi = b < 0 ? -1 : 0;
    it.b_lo = (uint64_t)b;
    it.c_hi = c < 0 ? -1 : 0;
    it.c_lo = (uint64_t)c;
    it.P0 = std::strtoull(argv[3], nullptr, 10);
    it.P1 = std::strtoull(argv[4], nullptr, 10);
    it.N0 = std::atoll(argv[5]);
    it.N1 = std::atoll(argv[6]);
    it.mod = argc > 7 ? std::strtoull(argv[7], nullptr, 10) : 1;
    it.res = argc > 8 ? std::strtoull(argv[8], nullptr, 10) : 0;
    const int threads = argc > 9 ? std::atoi(argv[9]) : (int)std::thread::hardware_concurrency();
    std::vector<ref_relation> rel(1 << 22);
    uint64_t np = 0;
    const auto t0 = std::chrono::steady_clock::now();
    const size_t n = ref_relations_threaded(it.P0, it.P1, &it, rel.data(), rel.size(), threads, 1ULL << 24, &np);
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (size_t i = 0; i < n && i < rel.size(); ++i)
        std::printf("%llu, %llu, %llu\n", (unsigned long long)rel[i].p, (unsigned long long)rel[i].M,
                    (unsigned long long)rel[i].q);
    std::fprintf(stderr, "primes=%llu relations=%zu seconds=%.3f threads=%d\n", (unsigned long long)np, n, s, threads);
    return 0;
}
#endif
