// driver.cpp -- the reference's GPU worker path, run as the GPU bar.
//
// BENCHMARK BASELINE ONLY (never the product).  The reference's GPU worker
// with GPU_sieve=1: for every chunk of the P range, CudaSiever::sieve_filter
// (Cuda.hpp:329-415) runs the reference's own kernels (psieve, prep_sv or
// prep_svq, bsgs_wg or bsgs_wq, collect; compiled from its Gpu.hpp by
// extract_kernels.py) and returns the numbers it could not rule out; then
// process_chunk's CPU check (Worker.hpp:222-280) keeps those that are prime
// (is_prime64) and solves each exactly (run_bsgs), on a pool of CPU threads
// while the GPU goes on with the next chunk (the reference's GPU feeder
// threads overlap the same way).  A chunk the GPU declines is sieved on the
// CPU, as the reference does without GPU_strict.  The host loop below
// restates sieve_filter with the runtime API; the number theory, the
// class-split rule (gpu_classes) and every size constant are the
// reference's own (Math.hpp, Sieve.hpp, compiled unmodified with the Boost
// shim of oracle/shim).
#include "Sieve.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

using namespace siever;

extern "C" {
typedef unsigned long long u64r;
int refk_psieve(unsigned, u64r, u64r, const unsigned*, unsigned, unsigned, u64r*, unsigned*, unsigned, cudaStream_t);
int refk_prep(int, unsigned, const u64r*, unsigned char*, u64r*, unsigned*, unsigned, u64r, long long, u64r, u64r,
              u64r, u64r, u64r, uint32_t, cudaStream_t);
int refk_bsgs(int, unsigned, const u64r*, unsigned char*, uint32_t, size_t, cudaStream_t);
int refk_collect(unsigned, const u64r*, const unsigned char*, uint32_t, u64r*, unsigned*, cudaStream_t);

typedef struct refgpu_item {
    int64_t b_hi;
    uint64_t b_lo;
    int64_t c_hi;
    uint64_t c_lo;
    uint64_t P0, P1;
    int64_t N0, N1;
    uint64_t mod, res;
} refgpu_item;

typedef struct refgpu_relation {
    uint64_t p, M, q;
} refgpu_relation;

typedef struct refgpu_stats {
    double seconds;          // wall time of the whole item
    double gpu_ms;           // device time of the sieve_filter passes (CUDA events)
    uint64_t flagged;        // numbers the GPU could not rule out
    uint64_t declined;       // chunks sieved on the CPU instead
} refgpu_stats;
}

namespace {

WorkItem to_work_item(const refgpu_item* it) {
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

// Device buffers of sieve_filter (Cuda.hpp:351-363), allocated once.
struct Buffers {
    unsigned* sp = nullptr;
    u64r* surv = nullptr;
    unsigned char* flags = nullptr;
    u64r* ent = nullptr;
    u64r* out = nullptr;
    unsigned* cnt = nullptr;       // survivors, entries, flagged
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    size_t smem_limit = 48 * 1024;
};

bool setup(Buffers& B) {
    const std::vector<uint32_t>& sp = gpu_sieve_primes();
    const size_t cap = kGpuSieveSurvCap;
    return cudaStreamCreate(&B.s) == cudaSuccess && cudaEventCreate(&B.e0) == cudaSuccess &&
           cudaEventCreate(&B.e1) == cudaSuccess &&
           cudaMalloc((void**)&B.sp, sp.size() * sizeof(unsigned)) == cudaSuccess &&
           cudaMalloc((void**)&B.surv, cap * sizeof(u64r)) == cudaSuccess &&
           cudaMalloc((void**)&B.flags, cap) == cudaSuccess &&
           cudaMalloc((void**)&B.ent, kGpuSieveEntBytes) == cudaSuccess &&
           cudaMalloc((void**)&B.out, cap * sizeof(u64r)) == cudaSuccess &&
           cudaMalloc((void**)&B.cnt, 3 * sizeof(unsigned)) == cudaSuccess &&
           cudaMemcpy(B.sp, sp.data(), sp.size() * sizeof(unsigned), cudaMemcpyHostToDevice) == cudaSuccess;
}

// CudaSiever::sieve_filter restated: false = declined (the caller sieves the chunk on the CPU).
bool sieve_filter(Buffers& B, uint64_t lo0, uint64_t hi, const WorkItem& item, std::vector<uint64_t>& flagged,
                  double* gpu_ms) {
    const uint64_t lo = lo0 | 1ULL;
    if (lo >= hi) return true;
    const uint64_t count = (hi - lo + 1) / 2;
    const uint64_t N0 = item.N0 < 0 ? 0 : (uint64_t)item.N0;
    const uint64_t N1 = (uint64_t)item.N1;
    const uint64_t cm = item.cls_mod == 0 ? 1 : item.cls_mod;
    uint64_t Qc = 0;
    std::vector<uint32_t> classes;
    const bool qmode = gpu_classes(item, Qc, classes);           // GPU_classes=1 (the default)
    const uint64_t kmax = qmode ? 0 : (N1 - N0) / cm + 2;
    uint64_t m = (uint64_t)std::sqrt((double)kmax) + 2;
    if (qmode) m = gpu_classes_max_m(item, Qc);
    unsigned tbits = 4;
    while ((1ULL << tbits) < m + m / 4) ++tbits;
    const size_t lbytes = (size_t(1) << tbits) * sizeof(uint32_t);
    if (lbytes + 1024 > B.smem_limit || tbits > 14) return false;
    const unsigned cap = kGpuSieveSurvCap, ent_cap = qmode ? kGpuSieveEntCapQ : kGpuSieveEntCap;
    const unsigned nsp = (unsigned)gpu_sieve_primes().size(), nsmall = gpu_sieve_nsmall();
    const u64r b = (u64r)(uint64_t)item.b;
    const long long c = (long long)item.c;
    std::vector<uint64_t> buf;
    for (uint64_t pb = 0; pb < count; pb += kGpuSievePassOdds) {
        const uint64_t pc = std::min<uint64_t>(kGpuSievePassOdds, count - pb);
        const uint64_t plo = lo + 2 * pb;
        unsigned h[3] = {0, 0, 0};
        cudaEventRecord(B.e0, B.s);
        if (cudaMemsetAsync(B.cnt, 0, 3 * sizeof(unsigned), B.s) != cudaSuccess) return false;
        const unsigned groups = (unsigned)((pc + kGpuSieveSegOdds - 1) / kGpuSieveSegOdds);
        if (refk_psieve(groups, plo, pc, B.sp, nsp, nsmall, B.surv, B.cnt, cap, B.s)) return false;
        if (cudaMemcpyAsync(h, B.cnt, sizeof(unsigned), cudaMemcpyDeviceToHost, B.s) != cudaSuccess ||
            cudaStreamSynchronize(B.s) != cudaSuccess)
            return false;
        const unsigned n = h[0];
        if (n > cap) return false;                                   // only for tiny p: the CPU path
        if (n != 0) {
            const unsigned blocks = (n + 63) / 64;
            if (refk_prep(qmode, blocks, B.surv, B.flags, B.ent, B.cnt + 1, ent_cap, b, c, N0, N1, cm, item.cls_res, Qc,
                          n, B.s))
                return false;
            if (cudaMemcpyAsync(h + 1, B.cnt + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, B.s) != cudaSuccess ||
                cudaStreamSynchronize(B.s) != cudaSuccess)
                return false;
            const unsigned n_ent = std::min(h[1], ent_cap);            // past ent_cap: flagged 2 by prep
            if (n_ent > 0 && refk_bsgs(qmode, n_ent, B.ent, B.flags, tbits, lbytes, B.s)) return false;
            if (refk_collect(blocks, B.surv, B.flags, n, B.out, B.cnt + 2, B.s)) return false;
            if (cudaMemcpyAsync(h + 2, B.cnt + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, B.s) != cudaSuccess ||
                cudaStreamSynchronize(B.s) != cudaSuccess)
                return false;
            if (h[2] > 0) {
                buf.resize(h[2]);
                if (cudaMemcpy(buf.data(), B.out, buf.size() * sizeof(u64r), cudaMemcpyDeviceToHost) != cudaSuccess)
                    return false;
                flagged.insert(flagged.end(), buf.begin(), buf.end());
            }
        }
        cudaEventRecord(B.e1, B.s);
        cudaEventSynchronize(B.e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, B.e0, B.e1);
        *gpu_ms += ms;
    }
    return true;
}

struct Job {
    uint64_t lo, hi;
    bool on_cpu;
    std::vector<uint64_t> flagged;
};

}  // namespace

extern "C" int refgpu_relations(int device, const refgpu_item* it, uint64_t chunk, int threads, refgpu_relation* out,
                                size_t cap, size_t* n_out, refgpu_stats* st) {
    static std::mutex once;
    static Buffers B;
    static bool ready = false;
    {
        std::lock_guard<std::mutex> g(once);
        if (!ready) {
            if (cudaSetDevice(device) != cudaSuccess || !setup(B)) return -1;
            ready = true;
        }
    }
    cudaSetDevice(device);
    const WorkItem item = to_work_item(it);
    const std::vector<uint32_t> small = sieve_small_primes(sieve_limit_for(item));
    const auto t0 = std::chrono::steady_clock::now();
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job> queue;
    bool producer_done = false;
    std::vector<Relation> rel;
    std::atomic<uint64_t> flagged_total{0}, declined{0};
    std::vector<std::thread> pool;
    if (threads < 1) threads = 1;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            std::vector<Relation> mine;
            for (;;) {
                Job job;
                {
                    std::unique_lock<std::mutex> lk(mu);
                    cv.wait(lk, [&] { return !queue.empty() || producer_done; });
                    if (queue.empty()) break;
                    job = std::move(queue.front());
                    queue.pop_front();
                }
                std::vector<uint64_t> ps;
                if (job.on_cpu) {
                    segmented_sieve((UInt128)job.lo, (UInt128)job.hi, small, ps);
                } else {
                    std::sort(job.flagged.begin(), job.flagged.end());
                    job.flagged.erase(std::unique(job.flagged.begin(), job.flagged.end()), job.flagged.end());
                    for (uint64_t p : job.flagged)
                        if (p >= job.lo && p < job.hi && is_prime64(p)) ps.push_back(p);
                }
                std::mt19937_64 rng(static_cast<uint64_t>(t + 1) ^ job.lo);
                for (uint64_t p : ps) {
                    Relation r;
                    if (run_bsgs(p, item, r, rng)) mine.push_back(r);
                }
            }
            std::lock_guard<std::mutex> g(mu);
            rel.insert(rel.end(), mine.begin(), mine.end());
        });
    double gpu_ms = 0;
    for (uint64_t lo = it->P0; lo < it->P1;) {
        const uint64_t hi = it->P1 - lo > chunk ? lo + chunk : it->P1;
        Job job{lo, hi, false, {}};
        const bool gpu_ok = hi < (1ULL << 62) && lo > 3 && sieve_filter(B, lo, hi, item, job.flagged, &gpu_ms);
        if (!gpu_ok) {
            job.on_cpu = true;
            job.flagged.clear();
            ++declined;
        }
        flagged_total += job.flagged.size();
        {
            std::lock_guard<std::mutex> g(mu);
            queue.push_back(std::move(job));
        }
        cv.notify_one();
        lo = hi;
    }
    {
        std::lock_guard<std::mutex> g(mu);
        producer_done = true;
    }
    cv.notify_all();
    for (std::thread& th : pool) th.join();
    std::sort(rel.begin(), rel.end(), [](const Relation& x, const Relation& y) { return x.p < y.p; });
    if (st) {
        st->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        st->gpu_ms = gpu_ms;
        st->flagged = flagged_total.load();
        st->declined = declined.load();
    }
    if (n_out) *n_out = rel.size();
    if (rel.size() > cap) return -3;
    for (size_t k = 0; k < rel.size(); ++k) out[k] = refgpu_relation{rel[k].p, rel[k].M, rel[k].q};
    return 0;
}
