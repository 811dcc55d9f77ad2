// siever_main.cpp -- mps_siever: the drop-in program around the B200 GPU path.
//
// Run in a directory holding prime.ini and worktodo.txt, like the
// reference's main() (Siever.cpp:75-212): for every Factor= item it resumes
// from core_<id>.p checkpoints (Worker.hpp:369-463), sieves [P0, P1) on the
// GPU through libmps_b200.so in checkpointed chunks, merges the core files
// into relations.p (Worker.hpp:469-495), applies the relations to the
// exponents (Worker.hpp:527-559) and appends the item's entry to
// results.json (Results.hpp:72-140).  SIGINT/SIGTERM/SIGHUP stop after the
// current chunk with the checkpoint kept.
//
// Differences, all deliberate: the relations come back exact from the
// device (no CPU re-check); chunks are processed in increasing p and each
// completed chunk is also recorded in core_progress.txt, so a resume starts
// exactly where the last chunk ended (the reference resumes at the minimum
// of the core files' last p, which can skip an unfinished chunk of a thread
// that wrote no relation yet); relations.p is sorted by p (the reference's
// order depends on thread timing); there is no CPU sieving path, so a range
// the GPU path does not take (P1 > 2^62) stops the program with an error.
//
// `mps_siever --results-entry <relations file> <Factor line> <timestamp> [results.json]`
// prints the results.json entry of one item for given relations and, with a
// fourth argument, appends it to that file (used by the tests; no GPU needed).
#include "../../include/mps_gpu.h"
#include "siever_host.hpp"

#include <atomic>
#include <csignal>
#include <cstring>
#include <unistd.h>

using namespace mpsh;

namespace {

std::atomic<bool> g_shutdown{false};
extern "C" void on_signal(int) { g_shutdown.store(true); }

const char* kProgress = "core_progress.txt";

mps_item to_mps(const WorkItem& w, uint64_t P0, uint64_t P1) {
    mps_item m{};
    m.b_hi = (int64_t)(w.b >> 64);
    m.b_lo = (uint64_t)w.b;
    m.c_hi = (int64_t)(w.c >> 64);
    m.c_lo = (uint64_t)w.c;
    m.P0 = P0;
    m.P1 = P1;
    m.N0 = (int64_t)w.N0;
    m.N1 = (int64_t)w.N1;
    m.mod = w.cls_mod;
    m.res = w.cls_res;
    return m;
}

std::string core_path(int id) { return "core_" + std::to_string(id) + ".p"; }

// The exact progress record of this item: "<b> <c> <P0> <P1> <N0> <N1> <mod> <res> <p_done>"
// (P0 the item's original P0); every p below p_done has been sieved.
std::string progress_key(const WorkItem& it) {
    return to_string128(it.b) + ' ' + to_string128(it.c) + ' ' + to_string128(it.P0_original) + ' ' +
           to_string128(it.P1) + ' ' + to_string128(it.N0) + ' ' + to_string128(it.N1) + ' ' +
           std::to_string(it.cls_mod) + ' ' + std::to_string(it.cls_res);
}

bool read_progress(const WorkItem& it, i128* p_done) {
    std::ifstream in(kProgress);
    if (!in) return false;
    std::string line;
    if (!std::getline(in, line)) return false;
    const std::string key = progress_key(it) + ' ';
    if (line.compare(0, key.size(), key) != 0) return false;
    try {
        *p_done = parse128(trim(line.substr(key.size())));
    } catch (...) {
        return false;
    }
    return *p_done >= it.P0_original && *p_done <= it.P1;
}

void write_progress(const WorkItem& it, i128 p_done) {
    const std::string tmp = std::string(kProgress) + ".tmp";
    {
        std::ofstream out(tmp, std::ios::trunc);
        out << progress_key(it) << ' ' << to_string128(p_done) << '\n';
        out.flush();
        if (!out) log_fatal("Failed to write " + tmp);
    }
    if (std::rename(tmp.c_str(), kProgress) != 0) log_fatal(std::string("Failed to replace ") + kProgress);
}

// Core files are looked for at ids 0 .. kCoreScan - 1 (the reference stops at
// the second missing id in a row, Worker.hpp:373-380; scanning the whole
// range also finds the files of a reference run whose first workers wrote
// nothing).
constexpr int kCoreScan = 1024;

// Worker.hpp:369-463 (reference resume), then the exact progress record when present.
void read_checkpoint(WorkItem& item) {
    i128 new_p0 = item.P1;
    bool any = false;
    for (int id = 0; id < kCoreScan; ++id) {
        std::ifstream in(core_path(id));
        if (!in) continue;
        std::string line, last;
        while (std::getline(in, line))
            if (!line.empty()) last = line;
        if (last.empty()) continue;
        std::stringstream ss(last);
        unsigned long long p = 0;
        char comma = 0;
        if (ss >> p && ss >> comma && comma == ',' && (i128)p < new_p0) {
            new_p0 = (i128)p;
            any = true;
        }
    }
    i128 exact = 0;
    const bool have_exact = read_progress(item, &exact);
    if (have_exact && exact > item.P0) {
        new_p0 = exact;
        any = true;
    }
    if (!any) {
        log_info("No checkpoint found, starting from original P0.");
        return;
    }
    if (new_p0 <= item.P0) {
        log_info("Checkpoint not ahead of current P0, starting from original P0.");
        return;
    }
    item.P0 = new_p0;
    uint64_t restored = 0;
    for (int id = 0; id < kCoreScan; ++id) {
        std::ifstream in(core_path(id));
        if (!in) continue;
        std::vector<std::string> kept;
        std::string line;
        while (std::getline(in, line)) {
            if (line.empty()) continue;
            std::stringstream ss(line);
            unsigned long long p = 0;
            char comma = 0;
            if (ss >> p && ss >> comma && comma == ',' && (i128)p < new_p0) kept.push_back(line);
        }
        in.close();
        std::ofstream out(core_path(id), std::ios::trunc);
        if (!out) log_fatal("Failed to trim checkpoint file: " + core_path(id));
        for (const std::string& l : kept) out << l << '\n';
        restored += kept.size();
    }
    item.relations_restored = restored;
    log_info("Checkpoint recovered: new P0 = " + to_string128(item.P0) +
             ", relations restored = " + std::to_string(restored));
}

// Worker.hpp:469-495, except that the lines are written in increasing p
// (the reference concatenates the files, an order that depends on thread
// timing), so relations.p is the same file on every run.
void merge_core_files() {
    std::vector<std::pair<unsigned long long, std::string>> lines;
    for (int id = 0; id < kCoreScan; ++id) {
        std::ifstream core(core_path(id));
        if (!core) continue;
        std::string line;
        while (std::getline(core, line)) {
            if (line.empty()) continue;
            std::stringstream ss(line);
            unsigned long long p = 0;
            ss >> p;
            lines.emplace_back(p, line);
        }
    }
    std::stable_sort(lines.begin(), lines.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    std::ofstream merged("relations.p", std::ios::binary | std::ios::trunc);
    if (!merged) log_fatal("Failed to create relations.p");
    for (const auto& l : lines) merged << l.second << '\n';
    merged.flush();
    if (!merged) log_fatal("Failed while writing relations.p");
    merged.close();
    for (int id = 0; id < kCoreScan; ++id) std::remove(core_path(id).c_str());
}

std::string eta_text(std::chrono::steady_clock::time_point start, size_t done, size_t total) {
    if (done == 0) return "unknown";
    if (done >= total) return "complete";
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    const double rem = el / (double)done * (double)(total - done);
    std::string ts = utc_timestamp(std::time(nullptr) + (std::time_t)rem);
    for (size_t k = 11; k < 19 && k < ts.size(); ++k)
        if (ts[k] == ':') ts[k] = '-';               // "YYYY-MM-DD HH-MM-SS UTC+0" (Worker.hpp:104-112)
    return ts;
}

int results_entry_mode(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr,
                     "usage: mps_siever --results-entry <relations file> <Factor line> <timestamp> [results.json]\n");
        return 2;
    }
    const std::string tmp = "/tmp/mps_siever_item_" + std::to_string(getpid()) + ".txt";
    {
        std::ofstream w(tmp);
        w << argv[3] << '\n';
    }
    std::vector<WorkItem> items = load_worktodo(tmp);
    std::remove(tmp.c_str());
    const std::vector<Relation> rel = load_relations(argv[2]);
    const auto cand = apply_relations(items[0], rel);
    const JValue entry = results_entry(items[0], cand, argv[4]);
    std::string text;
    serialize(entry, text);
    std::printf("%s\n", text.c_str());
    if (argc > 5) append_results_json(argv[5], entry);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc > 1 && std::strcmp(argv[1], "--results-entry") == 0) return results_entry_mode(argc, argv);
    struct sigaction action{};
    action.sa_handler = on_signal;
    sigemptyset(&action.sa_mask);
    sigaction(SIGINT, &action, nullptr);
    sigaction(SIGTERM, &action, nullptr);
    sigaction(SIGHUP, &action, nullptr);
    const auto start = std::chrono::steady_clock::now();

    log_info("Mass Prime Siever (B200 sm_100a worker) starting");
    try {
        Logger::instance().init("siever.log");
    } catch (const std::exception& ex) {
        log_fatal(ex.what());
    }
    PrimeConfig cfg = load_prime_config("prime.ini");
    std::vector<WorkItem> items = load_worktodo("worktodo.txt");
    log_info("Loaded " + std::to_string(items.size()) + " work item(s)");
    log_info("CPU_count=" + std::to_string(cfg.cpu_count) + " MemoryAllowed=" + std::to_string(cfg.memory_allowed_mb) +
             " MB");
    if (cfg.use_gpu == 0) log_info("UseGPU=0 ignored: this worker sieves on the GPU only");
    log_info("GPU_backend, GPU_threads, GPU_sieve and GPU_classes are ignored: the B200 path always sieves, "
             "filters and solves on the device");

    mps_tuning tun;
    mps_tuning_default(&tun);
    mps_ctx* ctx = nullptr;
    const int orc = mps_open(cfg.gpu_device, &tun, &ctx);
    if (orc != MPS_OK) {
        if (cfg.gpu_strict) log_fatal("GPU_strict=1 but no usable GPU backend; not sieving on the CPU");
        log_fatal("No usable CUDA device (mps_open returned " + std::to_string(orc) + "); this worker has no CPU path");
    }
    log_info("GPU enabled (B200 sm_100a): device " + std::to_string(cfg.gpu_device) + ", libmps_b200 ABI " +
             std::to_string(mps_abi_version()));

    const int worker_id = 0;                  // one writer: core_0.p, the first file any resume looks at
    const uint64_t ref_chunk = (uint64_t)cfg.memory_allowed_mb * 1024ull * 1024ull / (uint64_t)std::max(1, cfg.cpu_count);
    const uint64_t chunk = std::min<uint64_t>(std::max<uint64_t>(ref_chunk, 1ull << 24), 1ull << 32);

    for (size_t wi = 0; wi < items.size(); ++wi) {
        if (g_shutdown.load()) {
            log_info("Shutdown requested, stopping before next work item.");
            break;
        }
        WorkItem& item = items[wi];
        log_info("Processing work item " + std::to_string(wi + 1) + "/" + std::to_string(items.size()) +
                 " b=" + to_string128(item.b) + " c=" + to_string128(item.c));
        std::remove("relations.p");
        read_checkpoint(item);
        if (item.P1 > ((i128)1 << 62) || item.P0 < 0)
            log_fatal("P range outside the GPU path (0 <= P0, P1 <= 2^62); this worker has no CPU path");
        const uint64_t P0 = (uint64_t)item.P0, P1 = (uint64_t)item.P1;
        const size_t total = (size_t)((P1 - P0 + chunk - 1) / chunk);
        log_info("Chunk size per task: " + std::to_string(chunk) + " integers, " + std::to_string(total) +
                 " total chunks queued");
        std::vector<mps_relation> buf(1 << 16);
        uint64_t total_rel = item.relations_restored;
        size_t done = 0;
        for (uint64_t lo = P0; lo < P1 && !g_shutdown.load(); lo = std::min(P1, lo + chunk)) {
            const uint64_t hi = P1 - lo > chunk ? lo + chunk : P1;
            mps_item m = to_mps(item, lo, hi);
            size_t n = 0;
            int rc = mps_item_relations(ctx, &m, buf.data(), buf.size(), &n);
            if (rc == MPS_E_CAPACITY) {
                buf.resize(n);
                rc = mps_take_relations(ctx, buf.data(), nullptr, buf.size(), &n);
            }
            if (rc != MPS_OK) {
                const std::string why = mps_last_error(ctx);
                if (cfg.gpu_strict)
                    log_fatal("GPU_strict=1: the GPU sieve declined the chunk starting at " + std::to_string(lo) +
                              " (" + why + "); stopping instead of sieving on the CPU");
                log_fatal("The GPU path failed on the chunk starting at " + std::to_string(lo) + ": " + why);
            }
            if (n) {
                std::FILE* f = std::fopen(core_path(worker_id).c_str(), "ab");
                if (!f) log_fatal("Failed to append to " + core_path(worker_id));
                for (size_t k = 0; k < n; ++k) {
                    const std::string line = relation_line(Relation{buf[k].p, buf[k].M, buf[k].q});
                    std::fwrite(line.data(), 1, line.size(), f);
                }
                std::fclose(f);
            }
            write_progress(item, (i128)hi);
            ++done;
            total_rel += n;
            char pct[32];
            std::snprintf(pct, sizeof(pct), "%.2f", total ? 100.0 * (double)done / (double)total : 100.0);
            log_info("global " + std::to_string(done) + "/" + std::to_string(total) + " chunks (" + pct + "%), +" +
                     std::to_string(n) + " relations, " + std::to_string(total_rel) + " total relations, ETA " +
                     eta_text(start, done, total));
        }
        if (g_shutdown.load()) {
            log_info("Shutdown: checkpoint preserved in core_*.p files");
            break;
        }
        log_info("Merging core files");
        merge_core_files();
        const std::vector<Relation> rel = load_relations("relations.p");
        log_info("Loaded " + std::to_string(rel.size()) + " relation(s)");
        const auto cand = apply_relations(item, rel);
        append_results_json("results.json", results_entry(item, cand, now_timestamp()));
        log_info(final_status(item, cand, std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count()));
        log_info("Finished work item " + std::to_string(wi + 1));
        std::remove(kProgress);
    }
    if (!g_shutdown.load())
        log_info("Siever completed successfully, total elapsed " +
                 format_elapsed(std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count()));
    mps_close(ctx);
    return 0;
}
