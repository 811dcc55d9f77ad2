// siever_main.cpp -- mps_siever: the drop-in program around the B200 GPU path.
//
// Run in a directory holding prime.ini and worktodo.txt, like the
// reference's program (Siever.cpp:75-212).  For every Factor= item it
// resumes from the core files (checkpoint.hpp), sieves [P0, P1) on the GPU
// through libmps_b200.so one chunk at a time, appends each chunk's relations
// to core_0.p and records the chunk in core_progress.txt, then merges the
// core files into relations.p, lists the candidate primes of every exponent
// and appends the item's entry to results.json (formats.hpp).  SIGINT,
// SIGTERM and SIGHUP stop the run after the current chunk with the
// checkpoint kept.
//
// Deliberate differences from the reference: the relations come back exact
// from the device (no CPU re-check); relations.p is written in increasing p
// (the reference's order depends on thread timing); resume also uses the
// exact progress record; there is no CPU sieving path, so a range the GPU
// path does not take, or a chunk the device declines, stops the program.
// With GPU_strict=1 a declined chunk ends the run the way the reference's
// does (Worker.hpp:229-235, 358-360): the INFO line naming the chunk, then
// FATAL "Worker pool failed".
//
// `mps_siever --results-entry <relations file> <Factor line> <timestamp> [results.json]`
// prints the results.json entry of one item for the given relations and,
// with a fifth argument, appends it to that file (no GPU needed; used by the
// tests).
//
// Built with -DMPS_SIEVER_FAULTS (the mps_siever_faults test binary only),
// two environment variables inject failures on the host:
//   MPS_SIEVER_DECLINE_CHUNK=k   the k-th chunk call (from 0) returns MPS_E_CUDA
//                                without reaching the device;
//   MPS_SIEVER_SIGNAL_AFTER=k    the program raises SIGINT after its k-th chunk.
#include "../../include/mps_gpu.h"
#include "checkpoint.hpp"
#include "formats.hpp"

#include <atomic>
#include <chrono>
#include <csignal>
#include <cstring>
#include <unistd.h>

using namespace mpsio;

namespace {

std::atomic<bool> g_stop{false};
extern "C" void on_signal(int) { g_stop.store(true); }

mps_item device_item(const WorkItem& w, uint64_t lo, uint64_t hi) {
    mps_item m{};
    m.b_hi = (int64_t)(w.b >> 64);
    m.b_lo = (uint64_t)w.b;
    m.c_hi = (int64_t)(w.c >> 64);
    m.c_lo = (uint64_t)w.c;
    m.P0 = lo;
    m.P1 = hi;
    m.N0 = (int64_t)w.N0;
    m.N1 = (int64_t)w.N1;
    m.mod = w.mod;
    m.res = w.res;
    return m;
}

#ifdef MPS_SIEVER_FAULTS
long env_index(const char* name) {
    const char* v = std::getenv(name);
    return v ? std::atol(v) : -1;
}
#endif

// One chunk's relations through the C-ABI (the whole chunk as one item).
int chunk_relations(mps_ctx* ctx, const WorkItem& it, uint64_t lo, uint64_t hi, std::vector<Relation>& out,
                    std::string* why) {
#ifdef MPS_SIEVER_FAULTS
    static long calls = 0;
    if (calls++ == env_index("MPS_SIEVER_DECLINE_CHUNK")) {
        *why = "injected failure (MPS_SIEVER_DECLINE_CHUNK)";
        return MPS_E_CUDA;
    }
#endif
    const mps_item m = device_item(it, lo, hi);
    std::vector<mps_relation> buf(1 << 14);
    size_t n = 0;
    int rc = mps_item_relations(ctx, &m, buf.data(), buf.size(), &n);
    if (rc == MPS_E_CAPACITY) {
        buf.resize(n);
        rc = mps_take_relations(ctx, buf.data(), nullptr, buf.size(), &n);
    }
    if (rc != MPS_OK) {
        *why = mps_last_error(ctx);
        return rc;
    }
    out.clear();
    for (size_t k = 0; k < n; ++k) out.push_back(Relation{buf[k].p, buf[k].M, buf[k].q});
    return MPS_OK;
}

// "YYYY-MM-DD HH-MM-SS UTC+0" of the projected end (Worker.hpp:104-112), or
// "unknown" / "complete".
std::string eta(std::chrono::steady_clock::time_point t0, size_t done, size_t total) {
    if (done == 0) return "unknown";
    if (done >= total) return "complete";
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::string s = utc_stamp(std::time(nullptr) + (std::time_t)(el / (double)done * (double)(total - done)));
    for (size_t k = 11; k < 19 && k < s.size(); ++k)
        if (s[k] == ':') s[k] = '-';
    return s;
}

int results_entry_mode(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr,
                     "usage: mps_siever --results-entry <relations file> <Factor line> <timestamp> [results.json]\n");
        return 2;
    }
    char tmpl[] = "/tmp/mps_siever_item_XXXXXX";
    const int fd = mkstemp(tmpl);
    if (fd < 0) return 2;
    const std::string line = std::string(argv[3]) + "\n";
    if (::write(fd, line.data(), line.size()) != (ssize_t)line.size()) return 2;
    ::close(fd);
    const std::vector<WorkItem> items = read_worktodo(tmpl);
    std::remove(tmpl);
    const auto cand = candidate_primes(items[0], read_relations(argv[2]));
    const std::string entry = results_entry(items[0], cand, argv[4]);
    std::printf("%s\n", entry.c_str());
    if (argc > 5) append_result(argv[5], entry);
    return 0;
}

int run() {
    const auto t0 = std::chrono::steady_clock::now();
    info("Mass Prime Siever (B200 sm_100a worker) starting");
    Log::get().open("siever.log");
    const PrimeConfig cfg = read_prime_ini("prime.ini");
    std::vector<WorkItem> items = read_worktodo("worktodo.txt");
    info("Loaded " + std::to_string(items.size()) + " work item(s)");
    info("CPU_count=" + std::to_string(cfg.cpu_count) + " MemoryAllowed=" + std::to_string(cfg.memory_allowed_mb) +
         " MB");
    if (cfg.use_gpu == 0) info("UseGPU=0 ignored: this worker sieves on the GPU only");
    info("GPU_backend, GPU_threads, GPU_sieve and GPU_classes are ignored: the B200 path always sieves, "
         "filters and solves on the device");

    mps_tuning tun;
    mps_tuning_default(&tun);
    mps_ctx* ctx = nullptr;
    const int orc = mps_open(cfg.gpu_device, &tun, &ctx);
    if (orc != MPS_OK) {
        if (cfg.gpu_strict) fatal("GPU_strict=1 but no usable GPU backend; not sieving on the CPU");
        fatal("No usable CUDA device (mps_open returned " + std::to_string(orc) + "); this worker has no CPU path");
    }
    info("GPU enabled (B200 sm_100a): device " + std::to_string(cfg.gpu_device) + ", libmps_b200 ABI " +
         std::to_string(mps_abi_version()));

    // chunk size: MemoryAllowed / CPU_count integers like the reference's
    // workers (Worker.hpp:152-157), at least 2^24 and at most 2^32
    const uint64_t share = (uint64_t)cfg.memory_allowed_mb * (1ull << 20) / (uint64_t)std::max(1, cfg.cpu_count);
    const uint64_t chunk = std::min<uint64_t>(std::max<uint64_t>(share, 1ull << 24), 1ull << 32);
#ifdef MPS_SIEVER_FAULTS
    const long signal_after = env_index("MPS_SIEVER_SIGNAL_AFTER");
    long chunks_run = 0;
#endif

    for (size_t wi = 0; wi < items.size(); ++wi) {
        if (g_stop.load()) {
            info("Shutdown requested, stopping before next work item.");
            break;
        }
        WorkItem& it = items[wi];
        info("Processing work item " + std::to_string(wi + 1) + "/" + std::to_string(items.size()) +
             " b=" + i128_text(it.b) + " c=" + i128_text(it.c));
        std::remove("relations.p");
        resume(it);
        if (it.P1 > ((i128)1 << 62) || it.P0 < 0)
            fatal("P range outside the GPU path (0 <= P0, P1 <= 2^62); this worker has no CPU path");
        const uint64_t P0 = (uint64_t)it.P0, P1 = (uint64_t)it.P1;
        const size_t total = (size_t)((P1 - P0 + chunk - 1) / chunk);
        info("Chunk size per task: " + std::to_string(chunk) + " integers, " + std::to_string(total) +
             " total chunks queued");
        uint64_t found = it.relations_restored;
        size_t done = 0;
        std::vector<Relation> rel;
        for (uint64_t lo = P0; lo < P1 && !g_stop.load();) {
            const uint64_t hi = P1 - lo > chunk ? lo + chunk : P1;
            std::string why;
            const int rc = chunk_relations(ctx, it, lo, hi, rel, &why);
            if (rc != MPS_OK) {
                if (cfg.gpu_strict) {
                    info("GPU_strict=1: the GPU sieve declined the chunk starting at " + std::to_string(lo) +
                         "; stopping instead of sieving on the CPU");
                    info("Decline reason: " + why);
                    fatal("Worker pool failed");
                }
                fatal("The GPU path declined the chunk starting at " + std::to_string(lo) + " (" + why +
                      "); this worker has no CPU path to fall back to");
            }
            append_core(0, rel);
            write_progress(it, (i128)hi);
            ++done;
            found += rel.size();
            char pct[32];
            std::snprintf(pct, sizeof(pct), "%.2f", total ? 100.0 * (double)done / (double)total : 100.0);
            info("global " + std::to_string(done) + "/" + std::to_string(total) + " chunks (" + pct + "%), +" +
                 std::to_string(rel.size()) + " relations, " + std::to_string(found) + " total relations, ETA " +
                 eta(t0, done, total));
            lo = hi;
#ifdef MPS_SIEVER_FAULTS
            if (chunks_run++ == signal_after) std::raise(SIGINT);
#endif
        }
        if (g_stop.load()) {
            info("Shutdown: checkpoint preserved in core_*.p files");
            break;
        }
        info("Merging core files");
        merge_core_files();
        const std::vector<Relation> all = read_relations("relations.p");
        info("Loaded " + std::to_string(all.size()) + " relation(s)");
        const auto cand = candidate_primes(it, all);
        append_result("results.json", results_entry(it, cand, utc_now()));
        info(final_status(it, cand, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()));
        info("Finished work item " + std::to_string(wi + 1));
        std::remove(kProgressFile);
    }
    if (!g_stop.load())
        info("Siever completed successfully, total elapsed " +
             hms(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()));
    mps_close(ctx);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc > 1 && std::strcmp(argv[1], "--results-entry") == 0) return results_entry_mode(argc, argv);
    struct sigaction sa {};
    sa.sa_handler = on_signal;
    sigemptyset(&sa.sa_mask);
    for (int sig : {SIGINT, SIGTERM, SIGHUP}) sigaction(sig, &sa, nullptr);
    try {
        return run();
    } catch (const std::exception& ex) {
        fatal(std::string("Unhandled exception: ") + ex.what());
    }
}
