// mps_capi.cu -- the C-ABI of include/mps_gpu.h over the sm_100a kernels.
//
// A context owns one CUDA stream and its device buffers (allocated on
// demand, grown when a chunk overflows them, freed by mps_close).  A chunk
// of the prime range runs as sieve -> prep -> BSGS -> order on that stream;
// in the default (persistent) mode the four kernels are queued back to back
// and the host waits once per chunk, for the relation count.
#include "../../include/mps_gpu.h"
#include "mps_item.cuh"
#include "mps_kernels.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

using namespace mps;

namespace {

constexpr u64 kTwo62 = 1ull << 62;

// Odd primes 3..65521 and their division constants.
struct HostTables {
    std::vector<u32> sp;
    std::vector<u64> rcp, inv;
    HostTables() {
        std::vector<bool> comp(65536, false);
        for (u32 i = 3; i < 65536; i += 2) {
            if (comp[i]) continue;
            sp.push_back(i);
            for (u64 j = (u64)i * i; j < 65536; j += 2 * i) comp[j] = true;
        }
        for (u32 q : sp) {
            rcp.push_back(~0ull / q);
            u64 x = q;                       // q^-1 mod 2^64 by Newton
            for (int k = 0; k < 6; ++k) x *= 2 - q * x;
            inv.push_back(x);
        }
    }
};

const HostTables& host_tables() {
    static const HostTables t;
    return t;
}

}  // namespace

// One launch configuration (what the autotuner chooses per item class): the
// BSGS table kind, its load (table kind 2), lanes per prime, chains per lane
// and warps per block, and the sieve's segment size.
struct LaunchCfg {
    u32 kind = 0, load_shift = kDefaultLoadShift, chains = 2, warps = 4, seg_words = kDefaultSegWords;
    u32 lanes = 32;     // lanes per prime (table kind 2: 32, or groups of 16 / 8 for p < 2^49)
    u32 fill = kDefaultFill;           // table kinds 0 and 3: keys per word x 256, at most
    u32 scale = kDefaultBabyScale;     // baby steps: ceil(sqrt(j range)) x scale / 256
    bool operator==(const LaunchCfg& o) const {
        return kind == o.kind && load_shift == o.load_shift && chains == o.chains && warps == o.warps &&
               seg_words == o.seg_words && lanes == o.lanes && fill == o.fill && scale == o.scale;
    }
    bool operator!=(const LaunchCfg& o) const { return !(*this == o); }
};

// A tuned configuration with the calibration that chose it.
struct TuneEntry {
    LaunchCfg cfg;
    double ns_per_prime = 0;       // BSGS device time per prime of the calibration slice
};

// Events bracketing the four kernels of a chunk or wave: [2k] before and
// [2k + 1] after stage k (0 sieve, 1 prep, 2 BSGS, 3 order).
constexpr int kStageEvents = 8;

// One of the two in-flight wave slots of the batched engine.
struct WaveSlot {
    cudaStream_t stream = nullptr;
    cudaEvent_t evk[kStageEvents] = {};   // around sieve, prep, BSGS, order
    u64* d_surv = nullptr;
    u32* d_surv_item = nullptr;
    u64 surv_cap = 0;
    Entry* d_ent = nullptr;
    u64 ent_cap = 0;
    RawRelation* d_rel = nullptr;
    RawRelation* h_rel = nullptr;     // pinned
    u64 rel_cap = 0;
    Counters* d_ctr = nullptr;
    Counters* h_ctr = nullptr;        // pinned
    WaveDesc* d_wave = nullptr;
    WaveDesc* h_wave = nullptr;       // pinned
    // captured wave graphs of this slot, one per launch shape (tables, configuration) seen
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        u32 tbits = 0;
        LaunchCfg cfg;
    };
    std::vector<Graph> graphs;
    const DevItem* graph_items = nullptr;     // the buffers the graphs were captured with
    const ItemState* graph_state = nullptr;
    bool busy = false;
    std::vector<std::pair<u64, u64>> ranges;   // (lo, hi) of each run in flight
    std::vector<u32> range_item;
};

struct mps_ctx {
    int device = 0;
    int num_sms = 148;
    size_t smem_optin = 227 * 1024;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evb0 = nullptr, evb1 = nullptr;
    cudaEvent_t evk[kStageEvents] = {};
    mps_tuning tun{};
    std::string err;
    bool poisoned = false;
    mps_stats stats{};

    u32* d_sp = nullptr;
    u64* d_rcp = nullptr;
    u64* d_inv = nullptr;
    Counters* d_ctr = nullptr;
    Counters* h_ctr = nullptr;      // pinned
    u64* d_surv = nullptr;
    u64 surv_cap = 0;
    u32* d_surv_item = nullptr;
    Entry* d_ent = nullptr;
    u64 ent_cap = 0;
    RawRelation* d_rel = nullptr;
    RawRelation* h_rel = nullptr;   // pinned
    u64 rel_cap = 0;
    DevItem* d_items = nullptr;
    u64 items_cap = 0;
    ItemState* d_state = nullptr;      // per-item progress, same capacity as d_items
    WaveSlot slot[2];
    bool slots_ready = false;
    std::vector<u64> item_K;           // K of each item on the device (table sizing)
    std::vector<LaunchCfg> item_cfg;     // BSGS configuration of each item on the device
    std::map<u64, TuneEntry> tuned;    // autotuned configurations by item class (tune_key)
    std::vector<RawRelation> last;     // relations of the last call (kept for mps_take_relations)

    SieveTables tables() const { return SieveTables{d_sp, d_rcp, d_inv}; }
};

namespace {

int fail(mps_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(mps_ctx* c, cudaError_t e, const char* what) {
    c->poisoned = (e == cudaErrorIllegalAddress || e == cudaErrorLaunchFailure || e == cudaErrorIllegalInstruction ||
                   e == cudaErrorMisalignedAddress || e == cudaErrorHardwareStackError);
    return fail(c, MPS_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
    } while (0)

// Adds the device time of each stage of a finished chunk or wave to the stats.
int add_stage_times(mps_ctx* c, cudaEvent_t const* ev) {
    float ms[kStageEvents / 2] = {0, 0, 0, 0};
    for (int k = 0; k < kStageEvents / 2; ++k) CK(cudaEventElapsedTime(&ms[k], ev[2 * k], ev[2 * k + 1]), "event time");
    c->stats.sieve_ms += ms[0];
    c->stats.prep_ms += ms[1];
    c->stats.bsgs_ms += ms[2];
    c->stats.order_ms += ms[3];
    c->stats.bsgs_launches += 1;
    return MPS_OK;
}

template <class T>
int ensure(mps_ctx* c, T** ptr, u64* cap, u64 need, const char* what) {
    if (*cap >= need && *ptr) return MPS_OK;
    if (*ptr) CK(cudaFree(*ptr), "cudaFree");
    *ptr = nullptr;
    *cap = 0;
    CK(cudaMalloc((void**)ptr, need * sizeof(T)), what);
    *cap = need;
    return MPS_OK;
}

int ensure_rel(mps_ctx* c, u64 need) {
    if (c->rel_cap >= need && c->d_rel) return MPS_OK;
    if (c->d_rel) CK(cudaFree(c->d_rel), "cudaFree");
    if (c->h_rel) CK(cudaFreeHost(c->h_rel), "cudaFreeHost");
    c->d_rel = nullptr;
    c->h_rel = nullptr;
    c->rel_cap = 0;
    CK(cudaMalloc((void**)&c->d_rel, need * sizeof(RawRelation)), "relation buffer");
    CK(cudaMallocHost((void**)&c->h_rel, need * sizeof(RawRelation)), "pinned relation buffer");
    c->rel_cap = need;
    return MPS_OK;
}

u32 load_shift_of(const mps_ctx* c) { return c->tun.load_shift ? std::min<u32>(c->tun.load_shift, 4) : kDefaultLoadShift; }

// The configuration the tuning fields ask for.
LaunchCfg default_cfg(const mps_ctx* c) {
    LaunchCfg g;
    g.kind = c->tun.table_kind;
    g.load_shift = load_shift_of(c);
    g.chains = c->tun.chains ? c->tun.chains : 2;
    g.warps = c->tun.bsgs_warps ? c->tun.bsgs_warps : 4;
    const u32 lanes = c->tun.lanes;
    // groups of lanes exist for the 16-bit slot table with 1 or 2 chains
    g.lanes = g.kind == 2 && g.chains <= 2 && (lanes == 8 || lanes == 16) ? lanes : 32;
    g.fill = c->tun.table_fill ? std::min<u32>(c->tun.table_fill, 256) : kDefaultFill;
    g.scale = c->tun.baby_scale ? std::min<u32>(c->tun.baby_scale, 1024) : kDefaultBabyScale;
    return g;
}

// Item class of the autotuner: the bit length of K (the in-class exponent
// count, which sets the baby/giant split), the class modulus (which sets the
// power-residue split, capped at 4095) and the decimal digits of P0 (prime
// density, and FP64 or integer arithmetic).
u64 tune_key(u64 K, u64 cm, u64 P0) {
    u64 kb = 0;
    while ((K >> kb) != 0) ++kb;
    u64 pd = 0;
    for (u64 x = P0; x >= 10; x /= 10) ++pd;
    return (kb << 40) | (std::min<u64>(cm, 4095) << 8) | pd;
}

// The configuration for an item: the tuned one of its class, else the default.
LaunchCfg cfg_for(const mps_ctx* c, u64 K, u64 cm, u64 P0) {
    auto it = c->tuned.find(tune_key(K, cm, P0));
    return it != c->tuned.end() ? it->second.cfg : default_cfg(c);
}

// log2 of the primes a warp solves at once (lanes per prime 32, 16 or 8).
u32 groups_log(const LaunchCfg& g) { return g.kind == 2 ? (g.lanes == 8 ? 2 : g.lanes == 16 ? 1 : 0) : 0; }

// Keys a prime's table holds under configuration g with 4 << tb bytes per warp
// (fingerprint words: at most fill/256 keys per word on average).
u32 table_holds(const LaunchCfg& g, u32 tb) {
    const u32 fill = g.fill - 1 < 256 ? g.fill : 256;
    if (g.kind == 0) return std::max<u32>(((1u << (tb - 1)) * fill) >> 8, 1);
    if (g.kind == 2) return std::max<u32>(1u << (tb + 1 - g.load_shift) >> groups_log(g), 1);
    if (g.kind == 3) return std::max<u32>(((1u << (tb - 1)) * fill) >> 8, 1);      // the words of kind 0
    return std::max<u32>((1u << tb) / 5, 1);
}

// Room for a prime's keys (load at most 1/2 in 16-bit slots): fingerprint
// words hold four keys each, 32-bit slots one.
u32 table_room(const LaunchCfg& g, u32 tb) {
    if (g.kind == 0 || g.kind == 3) return 1u << tb;
    if (g.kind == 2) return (1u << tb) >> groups_log(g);
    return (1u << tb) - 1;
}

// Baby-step table size for an item: 4 << tbits bytes per warp, at most
// 8 KB by default (keeps ~24 warps resident per SM).  Every prime's j-range
// is at most K, so m_opt = ceil(sqrt(K)) x scale/256 baby steps is the most a
// prime of the item asks for; a wider N range than the table holds trades
// baby steps for giant steps.  Fingerprint words (table kinds 0 and 3):
// 2^(tbits-1) words of four keys, filled to at most fill/256 keys per word on
// average.  32-bit slots (table_kind 1): 2^tbits slots, load at most 1/5 (a
// probe then reads one slot).  16-bit slots (table_kind 2): 2^(tbits+1)
// slots, a prime's keys at most 2^-load_shift of them (up to 12 bits, 16 KB
// per warp, when load_shift > 2).
void table_for(const mps_ctx* c, const LaunchCfg& g, u64 K, u32* tbits, u32* max_baby) {
    const u64 m_sqrt = (u64)std::ceil(std::sqrt((double)std::max<u64>(K, 1)));
    const u64 m_opt = std::max<u64>(1, (m_sqrt * g.scale + 255) / 256);
    const u32 top = g.kind == 2 && g.load_shift > 2 ? 12 : 11;
    u32 tb = c->tun.table_bits;
    if (tb == 0) {
        tb = 6;
        while (table_holds(g, tb) < m_opt && tb < top) ++tb;
    }
    tb = std::min<u32>(std::max<u32>(tb, 6), 14);
    u32 mb = c->tun.max_baby ? c->tun.max_baby : table_holds(g, tb);
    mb = std::min<u32>(std::min<u32>(mb, kMaxBaby), table_room(g, tb));
    *tbits = tb;
    *max_baby = std::max<u32>(mb, 1);
}

// The baby-step cap of a launch with configuration g and tables of 4 << tbits
// bytes: no prime of the launch gets more, whatever its item's own sizing.
u32 launch_m_cap(const mps_ctx* c, const LaunchCfg& g, u32 tbits) {
    const u32 holds = c->tun.max_baby ? std::max(c->tun.max_baby, table_holds(g, tbits)) : table_holds(g, tbits);
    return std::max<u32>(1, std::min<u32>(std::min<u32>(holds, table_room(g, tbits)), kMaxBaby));
}

// Groups of lanes per prime run the FP64 solve only: a range that reaches
// 2^49 runs a whole warp per prime.
LaunchCfg for_range(LaunchCfg g, u64 hi) {
    if (hi > kFp64Limit) g.lanes = 32;
    return g;
}

// The device constants of an item (mps_item.cuh), with this context's split
// modulus, the item's BSGS configuration (tuned or default) and its
// baby-step sizing.
int make_dev_item(mps_ctx* c, const mps_item* it, u32 index, DevItem* d, LaunchCfg* cfg = nullptr) {
    const char* why = "";
    if (int r = item_constants(it, c->tun.class_modulus, index, d, &why)) return fail(c, r, why);
    const LaunchCfg g = cfg_for(c, d->K, d->cm, it->P0);
    u32 tb = 0, mb = 0;
    table_for(c, g, d->K, &tb, &mb);
    d->max_baby = mb;
    d->baby_scale = g.scale;
    if (cfg) *cfg = g;
    return MPS_OK;
}

u32 sieve_prime_count(u64 hi) {
    const std::vector<u32>& sp = host_tables().sp;
    u32 n = 0;
    while (n < sp.size() && (u64)sp[n] * sp[n] < hi) ++n;
    return n;
}

int reserve_items(mps_ctx* c, size_t n) {
    if (c->items_cap >= n && c->d_items) return MPS_OK;
    for (WaveSlot& w : c->slot)
        if (w.stream) CK(cudaStreamSynchronize(w.stream), "wave");
    if (c->d_state) CK(cudaFree(c->d_state), "cudaFree");
    c->d_state = nullptr;
    const u64 cap = std::max<u64>(n, 64);
    if (int r = ensure(c, &c->d_items, &c->items_cap, cap, "item buffer")) return r;
    CK(cudaMalloc((void**)&c->d_state, cap * sizeof(ItemState)), "item state");
    return MPS_OK;
}

int upload_items(mps_ctx* c, const DevItem* items, size_t n) {
    if (int r = reserve_items(c, std::max<size_t>(n, 1))) return r;
    CK(cudaMemcpyAsync(c->d_items, items, n * sizeof(DevItem), cudaMemcpyHostToDevice, c->stream), "item upload");
    CK(cudaMemsetAsync(c->d_state, 0, n * sizeof(ItemState), c->stream), "item state reset");
    CK(cudaStreamSynchronize(c->stream), "item upload");
    return MPS_OK;
}

int grid_for(mps_ctx* c, int per_sm) { return c->num_sms * per_sm; }

int bsgs_grid(mps_ctx* c, u32 tbits, u32 warps, u32 kind, int* grid) {
    const size_t smem = bsgs_smem_bytes(tbits, warps, kind);
    if (smem > c->smem_optin) return fail(c, MPS_E_ARG, "baby-step tables exceed shared memory");
    // blocks per SM limited by shared memory (1 KB reserved per block) and 64 warps per SM
    int per_sm = (int)(228 * 1024 / (smem + 1024));
    per_sm = std::min(per_sm, (int)(64 / warps));
    per_sm = std::max(per_sm, 1);
    *grid = c->num_sms * per_sm;
    return MPS_OK;
}

// Relations of the primes of one device chunk [lo, hi) (at most chunk_odds
// odd numbers) for item `item`, already on the device.  Appends RawRelations.
int run_chunk(mps_ctx* c, u64 lo, u64 hi, u32 item, u64 K, const LaunchCfg& g_item, std::vector<RawRelation>& out) {
    const LaunchCfg g = for_range(g_item, hi);
    const u64 lo_odd = std::max<u64>(lo, 3) | 1ull;
    const u64 n_odds = lo_odd < hi ? (hi - lo_odd + 1) / 2 : 0;
    const u32 include_two = (lo <= 2 && hi > 2) ? 1 : 0;
    if (n_odds == 0 && !include_two) return MPS_OK;
    const u64 chunk = c->tun.chunk_odds;
    const u64 need_surv = n_odds + 16;
    if (int r = ensure(c, &c->d_surv, &c->surv_cap, std::max<u64>(need_surv, chunk + 16), "survivor buffer")) return r;
    if (int r = ensure(c, &c->d_ent, &c->ent_cap, std::max<u64>(chunk / 4, 1 << 16), "entry buffer")) return r;
    if (int r = ensure_rel(c, std::max<u64>(c->rel_cap, 1 << 18))) return r;

    u32 tbits, max_baby;
    table_for(c, g, K, &tbits, &max_baby);
    (void)max_baby;
    const u32 warps = g.warps;

    SieveArgs sa{};
    sa.lo_odd = lo_odd;
    sa.n_odds = n_odds;
    sa.hi = hi;
    sa.include_two = include_two;
    sa.n_primes = sieve_prime_count(hi);
    sa.item = item;

    PrepArgs pa{};
    pa.surv = c->d_surv;
    pa.surv_cap = c->surv_cap;
    pa.surv_item = nullptr;
    pa.item0 = item;
    pa.items = c->d_items;
    pa.ent = c->d_ent;
    pa.ent_cap = c->ent_cap;
    pa.rel = c->d_rel;
    pa.rel_cap = c->rel_cap;
    pa.full_mr = c->tun.full_mr;
    pa.m_cap = launch_m_cap(c, g, tbits);
    pa.m_round = g.lanes * g.chains;
    pa.prime_below = kSievedPrimeBelow;             // survivors of the sieve

    BsgsArgs ba{};
    ba.ent = c->d_ent;
    ba.ent_cap = c->ent_cap;
    ba.rel = c->d_rel;
    ba.rel_cap = c->rel_cap;
    ba.tbits = tbits;
    ba.warps_per_block = warps;
    ba.chains = g.chains;
    ba.table_kind = g.kind;
    ba.fill = g.fill;
    ba.load_shift = g.load_shift;
    ba.lanes = g.lanes;
    ba.max_p = hi;

    OrderArgs oa{};
    oa.rel = c->d_rel;
    oa.rel_cap = c->rel_cap;
    oa.items = c->d_items;
    oa.tables = c->tables();

    cudaStream_t s = c->stream;
    CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(Counters), s), "counter reset");
    CK(cudaEventRecord(c->evk[0], s), "event");
    CK(launch_sieve(sa, c->tables(), c->d_surv, nullptr, c->surv_cap, c->d_ctr, s, g.seg_words), "sieve launch");
    CK(cudaEventRecord(c->evk[1], s), "event");
    int bgrid = 0;
    if (int r = bsgs_grid(c, tbits, warps, g.kind, &bgrid)) return r;
    if (c->tun.plain) {
        // the plain path: a host read of each stage's count sizes the next launch
        CK(cudaMemcpyAsync(c->h_ctr, c->d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s), "count read");
        CK(cudaStreamSynchronize(s), "sieve");
        const u64 ns = std::min<u64>(c->h_ctr->survivors, c->surv_cap);
        CK(cudaEventRecord(c->evk[2], s), "event");
        CK(launch_prep(pa, c->d_ctr, (int)std::max<u64>((ns + 255) / 256, 1), s), "prep launch");
        CK(cudaEventRecord(c->evk[3], s), "event");
        CK(cudaMemcpyAsync(c->h_ctr, c->d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s), "count read");
        CK(cudaStreamSynchronize(s), "prep");
        const u64 ne = std::min<u64>(c->h_ctr->entries, c->ent_cap);
        ba.persistent = 0;
        CK(cudaEventRecord(c->evk[4], s), "event");
        if (ne) CK(launch_bsgs(ba, c->d_ctr, (int)((ne + warps - 1) / warps), s), "bsgs launch");
        CK(cudaEventRecord(c->evk[5], s), "event");
    } else {
        CK(cudaEventRecord(c->evk[2], s), "event");
        CK(launch_prep(pa, c->d_ctr, grid_for(c, 16), s), "prep launch");
        CK(cudaEventRecord(c->evk[3], s), "event");
        ba.persistent = 1;
        CK(cudaEventRecord(c->evk[4], s), "event");
        CK(launch_bsgs(ba, c->d_ctr, bgrid, s), "bsgs launch");
        CK(cudaEventRecord(c->evk[5], s), "event");
    }
    CK(cudaEventRecord(c->evk[6], s), "event");
    CK(launch_order(oa, c->d_ctr, grid_for(c, 4), s), "order launch");
    CK(cudaEventRecord(c->evk[7], s), "event");
    CK(cudaMemcpyAsync(c->h_ctr, c->d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s), "count read");
    CK(cudaStreamSynchronize(s), "chunk");
    if (int r = add_stage_times(c, c->evk)) return r;
    c->stats.kernel_launches += 4;
    const Counters h = *c->h_ctr;
    if (h.status & (kStatusSurvivorOverflow | kStatusEntryOverflow)) {
        // a denser range than the buffers were sized for: halve the chunk
        if (n_odds <= 1024) return fail(c, MPS_E_CUDA, "device buffers overflow on a tiny chunk");
        const u64 mid = lo_odd + 2 * (n_odds / 2);
        if (int r = run_chunk(c, lo, mid, item, K, g, out)) return r;
        return run_chunk(c, mid, hi, item, K, g, out);
    }
    if (h.status & kStatusRelationOverflow) {
        if (int r = ensure_rel(c, std::max<u64>(2 * c->rel_cap, h.relations + 1024))) return r;
        return run_chunk(c, lo, hi, item, K, g, out);
    }
    if (h.status & kStatusOrderFailed) return fail(c, MPS_E_CUDA, "order computation did not factor p - 1");
    if (h.status & kStatusBadLaunch) return fail(c, MPS_E_CUDA, "a BSGS entry did not fit the launch's tables");
    const u64 nr = h.relations;
    if (nr) {
        CK(cudaMemcpyAsync(c->h_rel, c->d_rel, nr * sizeof(RawRelation), cudaMemcpyDeviceToHost, s), "relation read");
        CK(cudaStreamSynchronize(s), "relation read");
        for (u64 i = 0; i < nr; ++i)
            if (c->h_rel[i].q != ~0ull) out.push_back(c->h_rel[i]);
    }
    c->stats.odds += n_odds;
    c->stats.bsgs_steps += h.steps;
    c->stats.bsgs_baby_steps += h.baby;
    c->stats.survivors += h.survivors;
    c->stats.entries += h.entries;
    c->stats.chunks += 1;
    return MPS_OK;
}


// ------------------------------------------------------------ the wave engine --
//
// Items are cut into pieces of at most chunk_odds odd numbers; pieces are
// packed into waves of at most chunk_odds odd numbers in total (up to
// kMaxRuns runs, possibly of different items).  A wave runs as
//   H2D wave descriptor -> counters reset -> k_sieve_wave -> k_prep -> k_bsgs
//   -> k_order -> D2H counters + first relations
// on one of two slots (own stream and buffers), captured once per slot as a
// CUDA graph and replayed for every wave.  While the host reads wave k's
// results the device already runs wave k+1 on the other slot, so the tail of
// one wave's BSGS overlaps the next wave's sieve and prep.

constexpr u64 kGraphRelations = 4096;    // relations copied back inside the graph

void drop_graphs(WaveSlot& w) {
    for (WaveSlot::Graph& g : w.graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    w.graphs.clear();
}

int slot_alloc(mps_ctx* c, WaveSlot& w) {
    const u64 chunk = c->tun.chunk_odds;
    if (!w.stream) {
        CK(cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking), "stream");
        for (cudaEvent_t& ev : w.evk) CK(cudaEventCreate(&ev), "event");
        CK(cudaMalloc((void**)&w.d_ctr, sizeof(Counters)), "counters");
        CK(cudaMallocHost((void**)&w.h_ctr, sizeof(Counters)), "counters");
        CK(cudaMalloc((void**)&w.d_wave, sizeof(WaveDesc)), "wave descriptor");
        CK(cudaMallocHost((void**)&w.h_wave, sizeof(WaveDesc)), "wave descriptor");
    }
    if (w.surv_cap < chunk + kMaxRuns + 16) {
        if (w.d_surv) CK(cudaFree(w.d_surv), "cudaFree");
        if (w.d_surv_item) CK(cudaFree(w.d_surv_item), "cudaFree");
        w.surv_cap = chunk + kMaxRuns + 16;
        CK(cudaMalloc((void**)&w.d_surv, w.surv_cap * sizeof(u64)), "survivor buffer");
        CK(cudaMalloc((void**)&w.d_surv_item, w.surv_cap * sizeof(u32)), "survivor items");
        drop_graphs(w);
    }
    if (w.ent_cap < std::max<u64>(chunk / 4, 1 << 16)) {
        if (w.d_ent) CK(cudaFree(w.d_ent), "cudaFree");
        w.ent_cap = std::max<u64>(chunk / 4, 1 << 16);
        CK(cudaMalloc((void**)&w.d_ent, w.ent_cap * sizeof(Entry)), "entry buffer");
        drop_graphs(w);
    }
    if (w.rel_cap < (1u << 16)) {
        w.rel_cap = 1u << 16;
        CK(cudaMalloc((void**)&w.d_rel, w.rel_cap * sizeof(RawRelation)), "relation buffer");
        CK(cudaMallocHost((void**)&w.h_rel, w.rel_cap * sizeof(RawRelation)), "relation buffer");
    }
    return MPS_OK;
}

void slot_free(WaveSlot& w) {
    if (w.stream) cudaStreamSynchronize(w.stream);
    drop_graphs(w);
    for (void* p : {(void*)w.d_surv, (void*)w.d_surv_item, (void*)w.d_ent, (void*)w.d_rel, (void*)w.d_ctr,
                    (void*)w.d_wave})
        if (p) cudaFree(p);
    for (void* p : {(void*)w.h_rel, (void*)w.h_ctr, (void*)w.h_wave})
        if (p) cudaFreeHost(p);
    for (cudaEvent_t ev : w.evk)
        if (ev) cudaEventDestroy(ev);
    if (w.stream) cudaStreamDestroy(w.stream);
    w = WaveSlot();
}

// The per-wave launch sequence on the slot's stream (captured or direct).
int slot_enqueue(mps_ctx* c, WaveSlot& w, u32 tbits, const LaunchCfg& g, bool capturing) {
    const cudaStream_t s = w.stream;
    const u32 warps = g.warps;
    PrepArgs pa{};
    pa.surv = w.d_surv; pa.surv_cap = w.surv_cap; pa.surv_item = w.d_surv_item; pa.item0 = 0;
    pa.items = c->d_items; pa.ent = w.d_ent; pa.ent_cap = w.ent_cap; pa.rel = w.d_rel; pa.rel_cap = w.rel_cap;
    pa.full_mr = c->tun.full_mr;
    pa.m_cap = launch_m_cap(c, g, tbits);
    pa.m_round = g.lanes * g.chains;
    pa.prime_below = kSievedPrimeBelow;             // survivors of the sieve
    BsgsArgs ba{};
    ba.ent = w.d_ent; ba.ent_cap = w.ent_cap; ba.rel = w.d_rel; ba.rel_cap = w.rel_cap; ba.tbits = tbits;
    ba.warps_per_block = warps; ba.persistent = 1; ba.chains = g.chains;
    ba.table_kind = g.kind; ba.load_shift = g.load_shift; ba.lanes = g.lanes; ba.fill = g.fill;
    ba.max_p = 0;   // per-entry arithmetic
    OrderArgs oa{};
    oa.rel = w.d_rel; oa.rel_cap = w.rel_cap; oa.items = c->d_items; oa.tables = c->tables();
    int bgrid = 0;
    if (int r = bsgs_grid(c, tbits, warps, g.kind, &bgrid)) return r;
    CK(cudaMemcpyAsync(w.d_wave, w.h_wave, sizeof(WaveDesc), cudaMemcpyHostToDevice, s), "wave upload");
    CK(cudaMemsetAsync(w.d_ctr, 0, sizeof(Counters), s), "counter reset");
    // external records: a captured graph records these events on every replay
    const unsigned ev_flags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    CK(cudaEventRecordWithFlags(w.evk[0], s, ev_flags), "event");
    CK(launch_sieve_wave(w.d_wave, c->tables(), w.d_surv, w.d_surv_item, w.surv_cap, w.d_ctr, grid_for(c, 8), s,
                         g.seg_words),
       "sieve launch");
    CK(cudaEventRecordWithFlags(w.evk[1], s, ev_flags), "event");
    CK(cudaEventRecordWithFlags(w.evk[2], s, ev_flags), "event");
    CK(launch_prep(pa, w.d_ctr, grid_for(c, 16), s), "prep launch");
    CK(cudaEventRecordWithFlags(w.evk[3], s, ev_flags), "event");
    CK(cudaEventRecordWithFlags(w.evk[4], s, ev_flags), "event");
    CK(launch_bsgs(ba, w.d_ctr, bgrid, s), "bsgs launch");
    CK(cudaEventRecordWithFlags(w.evk[5], s, ev_flags), "event");
    CK(cudaEventRecordWithFlags(w.evk[6], s, ev_flags), "event");
    CK(launch_order(oa, w.d_ctr, grid_for(c, 4), s), "order launch");
    CK(cudaEventRecordWithFlags(w.evk[7], s, ev_flags), "event");
    CK(launch_commit(w.d_wave, w.d_rel, w.d_ctr, w.rel_cap, c->d_state, s), "commit launch");
    CK(cudaMemcpyAsync(w.h_ctr, w.d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s), "count read");
    CK(cudaMemcpyAsync(w.h_rel, w.d_rel, kGraphRelations * sizeof(RawRelation), cudaMemcpyDeviceToHost, s),
       "relation read");
    return MPS_OK;
}

int slot_launch(mps_ctx* c, WaveSlot& w, u32 tbits, const LaunchCfg& cfg) {
    if (c->tun.graphs_off) return slot_enqueue(c, w, tbits, cfg, false);
    if (w.graph_items != c->d_items || w.graph_state != c->d_state) {
        drop_graphs(w);
        w.graph_items = c->d_items;
        w.graph_state = c->d_state;
    }
    cudaGraphExec_t exec = nullptr;
    for (const WaveSlot::Graph& g : w.graphs)
        if (g.tbits == tbits && g.cfg == cfg) exec = g.exec;
    if (!exec) {
        if (w.graphs.size() >= 8) drop_graphs(w);
        CK(bsgs_reserve_smem(bsgs_smem_bytes(tbits, cfg.warps, cfg.kind)), "bsgs shared memory");
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(w.stream, cudaStreamCaptureModeThreadLocal), "capture");
        const int r = slot_enqueue(c, w, tbits, cfg, true);
        cudaError_t e = cudaStreamEndCapture(w.stream, &g);
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess) return cuda_fail(c, e, "end capture");
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(c, e, "graph instantiate");
        WaveSlot::Graph entry;
        entry.exec = exec;
        entry.tbits = tbits;
        entry.cfg = cfg;
        w.graphs.push_back(entry);
    }
    CK(cudaGraphLaunch(exec, w.stream), "graph launch");
    return MPS_OK;
}

// Numbers the segments of a wave's runs (segments of seg_words * 32 odd numbers).
void set_segments(WaveDesc* wave, u32 seg_words) {
    const u64 seg_odds = (u64)seg_words * 32;
    wave->total_segs = 0;
    for (u32 r = 0; r < wave->n_runs; ++r) {
        wave->runs[r].seg_begin = wave->total_segs;
        wave->total_segs += (wave->runs[r].n_odds + seg_odds - 1) / seg_odds;
    }
}

// The launch shape of a wave: the configuration of its item with the most
// in-class exponents (whose BSGS dominates the wave), with tables large
// enough for every item in it.
void wave_shape(const mps_ctx* c, const WaveSlot& w, u32* tbits, LaunchCfg* g) {
    u32 top = w.range_item[0];
    u64 hi = 0;
    for (u32 it : w.range_item)
        if (c->item_K[it] > c->item_K[top]) top = it;
    for (const auto& r : w.ranges) hi = std::max(hi, r.second);
    *g = for_range(c->item_cfg[top], hi);
    *tbits = 6;
    for (u32 it : w.range_item) {
        u32 tb, mb;
        table_for(c, *g, c->item_K[it], &tb, &mb);
        *tbits = std::max(*tbits, tb);
    }
}

// Waits for the slot's wave and appends its relations; on a buffer overflow
// the wave's runs are redone one by one on the chunk path (which splits them).
int slot_finish(mps_ctx* c, WaveSlot& w, std::vector<RawRelation>& out) {
    if (!w.busy) return MPS_OK;
    w.busy = false;
    CK(cudaStreamSynchronize(w.stream), "wave");
    const Counters h = *w.h_ctr;
    if (int r = add_stage_times(c, w.evk)) return r;
    c->stats.kernel_launches += 5;
    if (h.status & kStatusOrderFailed) return fail(c, MPS_E_CUDA, "order computation did not factor p - 1");
    if (h.status & kStatusBadLaunch) return fail(c, MPS_E_CUDA, "a BSGS entry did not fit the launch's tables");
    if (h.status & (kStatusSurvivorOverflow | kStatusEntryOverflow | kStatusRelationOverflow)) {
        // the commit kernel skipped this wave: redo its runs on the chunk path
        // (which splits or grows as needed) and record each in the item table
        for (size_t i = 0; i < w.ranges.size(); ++i) {
            std::vector<RawRelation> part;
            const u32 item = w.range_item[i];
            if (int r = run_chunk(c, w.ranges[i].first, w.ranges[i].second, item, c->item_K[item], c->item_cfg[item],
                                  part))
                return r;
            // the chunk path is done with its relation buffer: stage the run's relations there
            if (int r = ensure_rel(c, std::max<u64>(c->rel_cap, part.size()))) return r;
            if (!part.empty())
                CK(cudaMemcpyAsync(c->d_rel, part.data(), part.size() * sizeof(RawRelation), cudaMemcpyHostToDevice,
                                   c->stream),
                   "state update");
            CK(launch_state_add(c->d_state, item, w.ranges[i].second, c->d_rel, part.size(), c->stream), "state update");
            CK(cudaStreamSynchronize(c->stream), "state update");
            out.insert(out.end(), part.begin(), part.end());
        }
        return MPS_OK;
    }
    const u64 nr = h.relations;
    if (nr > kGraphRelations)
        CK(cudaMemcpy(w.h_rel + kGraphRelations, w.d_rel + kGraphRelations,
                      (nr - kGraphRelations) * sizeof(RawRelation), cudaMemcpyDeviceToHost),
           "relation read");
    for (u64 i = 0; i < nr; ++i)
        if (w.h_rel[i].q != ~0ull) out.push_back(w.h_rel[i]);
    c->stats.bsgs_steps += h.steps;
    c->stats.bsgs_baby_steps += h.baby;
    c->stats.survivors += h.survivors;
    c->stats.entries += h.entries;
    c->stats.chunks += 1;
    return MPS_OK;
}

// Relations of the items already on the device (d_items, item_K set), each
// over [lo_i, hi_i), through the double-buffered wave engine.
int run_waves(mps_ctx* c, const std::vector<u64>& lo, const std::vector<u64>& hi, std::vector<RawRelation>& out) {
    if (!c->slots_ready) {
        for (WaveSlot& w : c->slot)
            if (int r = slot_alloc(c, w)) return r;
        c->slots_ready = true;
    }
    for (WaveSlot& w : c->slot)
        if (int r = slot_alloc(c, w)) return r;
    const u64 chunk = c->tun.chunk_odds;
    int k = 0;
    WaveSlot* cur = nullptr;
    u64 wave_odds = 0;
    auto flush = [&]() -> int {
        if (!cur || cur->h_wave->n_runs == 0) return MPS_OK;
        u32 tbits;
        LaunchCfg g;
        wave_shape(c, *cur, &tbits, &g);
        set_segments(cur->h_wave, g.seg_words);
        if (int r = slot_launch(c, *cur, tbits, g)) return r;
        cur->busy = true;
        k ^= 1;
        cur = nullptr;
        wave_odds = 0;
        return MPS_OK;
    };
    for (size_t i = 0; i < lo.size(); ++i) {
        for (u64 a = lo[i]; a < hi[i];) {
            const u64 lo_odd = std::max<u64>(a, 3) | 1ull;
            if (!cur) {
                cur = &c->slot[k];
                if (int r = slot_finish(c, *cur, out)) return r;   // the slot's previous wave
                cur->h_wave->n_runs = 0;
                cur->ranges.clear();
                cur->range_item.clear();
            }
            const u64 room = chunk - wave_odds;
            u64 b = hi[i];
            if (lo_odd < hi[i] && (hi[i] - lo_odd + 1) / 2 > room) b = lo_odd + 2 * room;
            SieveRun& run = cur->h_wave->runs[cur->h_wave->n_runs++];
            run.lo_odd = lo_odd;
            run.n_odds = lo_odd < b ? (b - lo_odd + 1) / 2 : 0;
            run.include_two = (a <= 2 && b > 2) ? 1 : 0;
            run.n_primes = sieve_prime_count(b);
            run.item = (u32)i;
            run.pad = 0;
            run.hi = b;
            cur->ranges.push_back({a, b});
            cur->range_item.push_back((u32)i);
            wave_odds += run.n_odds;
            c->stats.odds += run.n_odds;
            a = b;
            if (wave_odds >= chunk || cur->h_wave->n_runs == kMaxRuns)
                if (int r = flush()) return r;
        }
    }
    if (int r = flush()) return r;
    for (int j = 0; j < 2; ++j)
        if (int r = slot_finish(c, c->slot[(k + j) & 1], out)) return r;
    return MPS_OK;
}


// ---------------------------------------------------------------- serving --
//
// A server owns a context and a worker thread.  Submitted items wait in a
// queue until admitted: an item is admitted while fewer than max_active items
// are in flight and the device memory its pieces need -- survivors and BSGS
// entries of one piece of its P range, plus its baby-step tables for the
// resident warps -- fits the budget left by the items already in flight.
// Every wave takes one piece from each in-flight item in turn (continuous
// batching: items admitted while others run join the next wave), so short
// items finish after a few waves while long ones keep going.  Each item's
// progress (P sieved, relations found) lives in a device table updated by
// the commit kernel at the end of every wave; relations are mirrored to the
// host as waves complete.

}  // namespace

struct ServeReq {
    u64 ticket = 0;
    mps_item item{};
    DevItem d{};
    int slot = -1;                     // device item index while in flight
    u64 cursor = 0;                    // next P to hand to a wave
    u32 inflight = 0;                  // waves in flight with a piece of this item
    std::multiset<u64> piece_lo;       // low ends of this item's pieces in flight
    u64 mem = 0;                       // device bytes its reservation takes (its relation buffer)
    u64 pool_off = 0;                  // the reservation's offset in the server's pool, while admitted
    bool relations_on_device = false;  // the result was read from the item's device buffer
    int state = 0;                     // 0 queued, 1 active, 2 done, 3 failed
    int error = 0;
    std::vector<RawRelation> rel;
    std::chrono::steady_clock::time_point t_submit, t_admit, t_done;
};

// First-fit allocator over a device pool [0, size), 256-byte granules; free
// blocks kept by offset and merged with their neighbours on release.
class PoolAlloc {
public:
    void reset(u64 size) {
        free_.clear();
        if (size) free_[0] = size;
        total_ = size;
        used_ = 0;
    }
    bool take(u64 bytes, u64* off) {
        bytes = (bytes + 255) & ~255ull;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const u64 rest = it->second - bytes, at = it->first + bytes;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used_ += bytes;
            return true;
        }
        return false;
    }
    void give(u64 off, u64 bytes) {
        bytes = (bytes + 255) & ~255ull;
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    u64 used() const { return used_; }
    u64 total() const { return total_; }

private:
    std::map<u64, u64> free_;
    u64 total_ = 0, used_ = 0;
};

struct mps_server {
    mps_ctx* ctx = nullptr;
    unsigned char* pool = nullptr;     // device memory the admitted items' reservations live in
    PoolAlloc alloc;
    mps_serve_config cfg{};
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<u64> queue;
    std::map<u64, ServeReq> reqs;
    std::vector<u64> slot_owner;       // device item slot -> ticket (0: free)
    u64 next_ticket = 1;
    u32 active = 0;
    bool stop = false;
    int fatal = 0;
    std::string fatal_msg;
    std::vector<u64> wave_tickets[2];  // tickets with a piece in each slot's wave
};

namespace {

double ms_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// The relations an item may give, for its device reservation: a prime p <= K
// (K in-class exponents) can meet a whole period of b's order, so each of
// those counts once; a larger p divides one of the K values with chance about
// K/p, and the sum of K/p over the primes of [a, b) is about
// K (ln ln b - ln ln a).  Twice that plus 256, at most 2^26.
u64 expected_relations(const DevItem& d, const mps_item& it) {
    const double K = (double)d.K;
    const auto approx_pi = [](double x) { return x < 3 ? 0.0 : x / std::log(x); };
    const double a = std::max<double>((double)it.P0, 2.0), b = (double)it.P1;
    const double split = std::min(b, std::max(a, K + 1));
    double e = split > a ? approx_pi(split) - approx_pi(a) : 0.0;
    const double lo = std::max(split, 3.0);
    if (b > lo) e += K * (std::log(std::log(b)) - std::log(std::log(lo)));
    return (u64)std::min(2.0 * e + 256.0, (double)(1ull << 26));
}

// Reads a finished item's relations from its device buffer; false when they
// did not all fit (the host copy of the wave results is used then).
bool read_device_relations(mps_server* sv, const ServeReq& q, std::vector<RawRelation>* out) {
    ItemState h{};
    if (cudaMemcpy(&h, sv->ctx->d_state + q.slot, sizeof(ItemState), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    if (!h.rel_buf || h.n_rel > h.rel_cap) return false;
    out->resize(h.n_rel);
    if (h.n_rel &&
        cudaMemcpy(out->data(), h.rel_buf, h.n_rel * sizeof(RawRelation), cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    std::sort(out->begin(), out->end(), [](const RawRelation& a, const RawRelation& b) { return a.p < b.p; });
    return true;
}

void serve_route(mps_server* sv, int k, std::vector<RawRelation>& rel, const WaveSlot& w) {
    for (size_t i = 0; i < w.ranges.size(); ++i) {
        auto it = sv->reqs.find(sv->slot_owner[w.range_item[i]]);
        if (it == sv->reqs.end()) continue;
        auto pos = it->second.piece_lo.find(w.ranges[i].first);
        if (pos != it->second.piece_lo.end()) it->second.piece_lo.erase(pos);
    }
    for (const RawRelation& r : rel) {
        const u64 t = sv->slot_owner[r.item];
        auto it = sv->reqs.find(t);
        if (it != sv->reqs.end()) it->second.rel.push_back(r);
    }
    for (u64 t : sv->wave_tickets[k]) {
        auto it = sv->reqs.find(t);
        if (it == sv->reqs.end()) continue;
        ServeReq& q = it->second;
        if (q.inflight) --q.inflight;
        if (q.state == 1 && q.inflight == 0 && q.cursor >= q.item.P1) {
            q.state = 2;
            q.t_done = std::chrono::steady_clock::now();
            std::sort(q.rel.begin(), q.rel.end(), [](const RawRelation& a, const RawRelation& b) { return a.p < b.p; });
            // the item's device-resident result; it must equal the waves' host copy
            std::vector<RawRelation> dev;
            if (read_device_relations(sv, q, &dev)) {
                const bool same = dev.size() == q.rel.size() &&
                                  std::equal(dev.begin(), dev.end(), q.rel.begin(), [](const RawRelation& a, const RawRelation& b) {
                                      return a.p == b.p && a.M == b.M && a.q == b.q;
                                  });
                if (same) {
                    q.rel.swap(dev);
                    q.relations_on_device = true;
                } else {
                    q.state = 3;
                    q.error = MPS_E_STATE;
                }
            }
            sv->slot_owner[q.slot] = 0;
            sv->alloc.give(q.pool_off, q.mem);
            --sv->active;
        }
    }
    sv->wave_tickets[k].clear();
}

void serve_fail_all(mps_server* sv, int code, const std::string& msg) {
    sv->fatal = code;
    sv->fatal_msg = msg;
    for (auto& kv : sv->reqs)
        if (kv.second.state < 2) {
            kv.second.state = 3;
            kv.second.error = code;
            kv.second.t_done = std::chrono::steady_clock::now();
        }
    sv->queue.clear();
}

void serve_loop(mps_server* sv) {
    mps_ctx* c = sv->ctx;
    cudaSetDevice(c->device);
    const u64 chunk = c->tun.chunk_odds;
    // every wave of the server has one launch shape: the default configuration
    // with the tables of the widest N range (launch_m_cap keeps every prime within them)
    const LaunchCfg cfg = default_cfg(c);
    u32 tbits = 11;
    {
        u32 mb;
        table_for(c, cfg, 10000000ull, &tbits, &mb);
    }
    int k = 0;
    std::unique_lock<std::mutex> lk(sv->mu);
    for (;;) {
        // admission: an item enters when a device slot is free and its
        // reservation fits in the pool; in arrival order
        while (!sv->queue.empty() && sv->active < sv->cfg.max_active) {
            ServeReq& q = sv->reqs[sv->queue.front()];
            int slot = -1;
            for (size_t i = 0; i < sv->slot_owner.size(); ++i)
                if (sv->slot_owner[i] == 0) {
                    slot = (int)i;
                    break;
                }
            if (slot < 0) break;
            u64 off = 0;
            if (!sv->alloc.take(q.mem, &off)) {
                if (sv->active > 0) break;                  // waits until a reservation is released
                // larger than the whole pool: it can never be admitted
                sv->queue.pop_front();
                q.state = 3;
                q.error = MPS_E_CAPACITY;
                q.t_done = std::chrono::steady_clock::now();
                sv->cv_done.notify_all();
                continue;
            }
            sv->queue.pop_front();
            q.slot = slot;
            q.pool_off = off;
            q.d.item_index = (u32)slot;
            sv->slot_owner[slot] = q.ticket;
            ++sv->active;
            q.state = 1;
            q.cursor = q.item.P0;
            q.t_admit = std::chrono::steady_clock::now();
            c->item_K[slot] = q.d.K;
            c->item_cfg[slot] = cfg;
            ItemState st{};
            st.rel_cap = q.mem / sizeof(RawRelation);
            st.rel_buf = reinterpret_cast<RawRelation*>(sv->pool + off);
            cudaError_t e = cudaMemcpy(c->d_items + slot, &q.d, sizeof(DevItem), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(c->d_state + slot, &st, sizeof(ItemState), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                serve_fail_all(sv, MPS_E_CUDA, std::string("item upload: ") + cudaGetErrorString(e));
                break;
            }
        }
        // pieces of every in-flight item with P left, round robin
        std::vector<ServeReq*> work;
        for (auto& kv : sv->reqs)
            if (kv.second.state == 1 && kv.second.cursor < kv.second.item.P1) work.push_back(&kv.second);
        const bool any_inflight = c->slot[0].busy || c->slot[1].busy;
        if (work.empty() && !any_inflight) {
            if (sv->stop && sv->queue.empty()) break;
            sv->cv_done.notify_all();
            sv->cv_work.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        WaveSlot& w = c->slot[k];
        // the slot's previous wave: wait without the lock, then route
        if (w.busy) {
            std::vector<RawRelation> rel;
            lk.unlock();
            const int r = slot_finish(c, w, rel);
            lk.lock();
            if (r) {
                serve_fail_all(sv, r, c->err);
                sv->cv_done.notify_all();
                break;
            }
            serve_route(sv, k, rel, w);
            sv->cv_done.notify_all();
        }
        if (!work.empty()) {
            w.h_wave->n_runs = 0;
            w.ranges.clear();
            w.range_item.clear();
            u64 wave_odds = 0;
            const u64 quantum = std::max<u64>(sv->cfg.piece_odds, chunk / std::max<size_t>(work.size(), 1));
            for (bool more = true; more && wave_odds < chunk && w.h_wave->n_runs < kMaxRuns;) {
                more = false;
                for (ServeReq* q : work) {
                    if (q->cursor >= q->item.P1 || wave_odds >= chunk || w.h_wave->n_runs >= kMaxRuns) continue;
                    const u64 a = q->cursor;
                    const u64 lo_odd = std::max<u64>(a, 3) | 1ull;
                    const u64 take = std::min<u64>(quantum, chunk - wave_odds);
                    u64 b = q->item.P1;
                    if (lo_odd < b && (b - lo_odd + 1) / 2 > take) b = lo_odd + 2 * take;
                    SieveRun& run = w.h_wave->runs[w.h_wave->n_runs++];
                    run.lo_odd = lo_odd;
                    run.n_odds = lo_odd < b ? (b - lo_odd + 1) / 2 : 0;
                    run.include_two = (a <= 2 && b > 2) ? 1 : 0;
                    run.n_primes = sieve_prime_count(b);
                    run.item = (u32)q->slot;
                    run.pad = 0;
                    run.hi = b;
                    w.ranges.push_back({a, b});
                    w.range_item.push_back((u32)q->slot);
                    wave_odds += run.n_odds;
                    c->stats.odds += run.n_odds;
                    q->cursor = b;
                    q->piece_lo.insert(a);
                    if (std::find(sv->wave_tickets[k].begin(), sv->wave_tickets[k].end(), q->ticket) ==
                        sv->wave_tickets[k].end()) {
                        sv->wave_tickets[k].push_back(q->ticket);
                        ++q->inflight;
                    }
                    if (q->cursor < q->item.P1) more = true;
                }
            }
            set_segments(w.h_wave, cfg.seg_words);
            const int r = slot_launch(c, w, tbits, cfg);
            if (r) {
                serve_fail_all(sv, r, c->err);
                sv->cv_done.notify_all();
                break;
            }
            w.busy = true;
        }
        k ^= 1;
    }
    sv->cv_done.notify_all();
}


int check_ctx(mps_ctx* c) {
    if (!c) return MPS_E_ARG;
    if (c->poisoned) return fail(c, MPS_E_STATE, "context poisoned by an earlier device fault: " + c->err);
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    return MPS_OK;
}

void begin_call(mps_ctx* c) {
    std::memset(&c->stats, 0, sizeof(c->stats));
    cudaEventRecord(c->ev0, c->stream);
}

int end_call(mps_ctx* c) {
    CK(cudaEventRecord(c->ev1, c->stream), "event");
    CK(cudaEventSynchronize(c->ev1), "event sync");
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1), "event time");
    c->stats.device_ms = ms;
    return MPS_OK;
}

// [lo, hi) in device chunks of at most chunk_odds odd numbers.
int run_range(mps_ctx* c, u64 lo, u64 hi, u32 item, u64 K, const LaunchCfg& g, std::vector<RawRelation>& rel) {
    const u64 chunk = c->tun.chunk_odds;
    for (u64 a = lo; a < hi;) {
        const u64 lo_odd = std::max<u64>(a, 3) | 1ull;
        u64 b = hi;
        if (lo_odd < hi && (hi - lo_odd + 1) / 2 > chunk) b = lo_odd + 2 * chunk;
        if (int r = run_chunk(c, a, b, item, K, g, rel)) return r;
        a = b;
    }
    return MPS_OK;
}

int relations_of(mps_ctx* c, const mps_item* item, u64 lo, u64 hi, std::vector<RawRelation>& rel) {
    DevItem d;
    LaunchCfg g;
    if (int r = make_dev_item(c, item, 0, &d, &g)) return r;
    if (lo >= hi) return MPS_OK;
    if (hi > kTwo62) return fail(c, MPS_E_RANGE, "hi must not exceed 2^62");
    if (int r = upload_items(c, &d, 1)) return r;
    return run_range(c, lo, hi, 0, d.K, g, rel);
}

void sort_by_p(std::vector<RawRelation>& rel) {
    std::sort(rel.begin(), rel.end(), [](const RawRelation& a, const RawRelation& b) {
        return a.item != b.item ? a.item < b.item : a.p < b.p;
    });
}

int copy_out(mps_ctx* c, const std::vector<RawRelation>& rel, mps_relation* out, uint32_t* out_item, size_t cap,
             size_t* n_out) {
    if (n_out) *n_out = rel.size();
    c->stats.relations = rel.size();
    if (&rel != &c->last) c->last = rel;
    if (rel.size() > cap) return fail(c, MPS_E_CAPACITY, "output buffer too small (mps_take_relations returns them)");
    for (size_t i = 0; i < rel.size(); ++i) {
        out[i].p = rel[i].p;
        out[i].M = rel[i].M;
        out[i].q = rel[i].q;
        if (out_item) out_item[i] = rel[i].item;
    }
    return MPS_OK;
}

}  // namespace

extern "C" {

int mps_abi_version(void) { return MPS_ABI_VERSION; }

int mps_tuning_default(mps_tuning* t) {
    if (!t) return MPS_E_ARG;
    std::memset(t, 0, sizeof(*t));
    t->struct_size = sizeof(mps_tuning);
    t->chunk_odds = 1ull << 26;
    t->bsgs_warps = 4;
    t->table_kind = 3;          // fingerprint words with count-byte claims (fastest measured on the B200)
    return MPS_OK;
}

int mps_open(int device, const mps_tuning* tuning, mps_ctx** out) {
    if (!out) return MPS_E_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return MPS_E_NODEV;
    if (device < 0 || device >= count) return MPS_E_NODEV;
    mps_ctx* c = new mps_ctx();
    c->device = device;
    mps_tuning_default(&c->tun);
    if (tuning) {
        if (tuning->struct_size != sizeof(mps_tuning)) {
            delete c;
            return MPS_E_ARG;
        }
        const mps_tuning d = c->tun;
        c->tun = *tuning;
        if (!c->tun.chunk_odds) c->tun.chunk_odds = d.chunk_odds;
        if (!c->tun.bsgs_warps) c->tun.bsgs_warps = d.bsgs_warps;
    }
    if (c->tun.chunk_odds < 4096) c->tun.chunk_odds = 4096;
    if (c->tun.bsgs_warps > 8) c->tun.bsgs_warps = 8;       // the BSGS kernel is built for <= 256 threads per block
    auto bail = [&](cudaError_t e, const char* what) {
        fprintf(stderr, "mps_open: %s: %s\n", what, cudaGetErrorString(e));
        mps_close(c);
        return MPS_E_CUDA;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(e, "cudaSetDevice");
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) return bail(e, "properties");
    c->num_sms = prop.multiProcessorCount;
    c->smem_optin = prop.sharedMemPerBlockOptin;
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    for (cudaEvent_t* ev : {&c->ev0, &c->ev1, &c->evb0, &c->evb1})
        if ((e = cudaEventCreate(ev)) != cudaSuccess) return bail(e, "event");
    for (cudaEvent_t& ev : c->evk)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) return bail(e, "event");
    const HostTables& t = host_tables();
    const size_t n = t.sp.size();
    if ((e = cudaMalloc((void**)&c->d_sp, n * sizeof(u32))) != cudaSuccess) return bail(e, "tables");
    if ((e = cudaMalloc((void**)&c->d_rcp, n * sizeof(u64))) != cudaSuccess) return bail(e, "tables");
    if ((e = cudaMalloc((void**)&c->d_inv, n * sizeof(u64))) != cudaSuccess) return bail(e, "tables");
    if ((e = cudaMalloc((void**)&c->d_ctr, sizeof(Counters))) != cudaSuccess) return bail(e, "counters");
    if ((e = cudaMallocHost((void**)&c->h_ctr, sizeof(Counters))) != cudaSuccess) return bail(e, "counters");
    if ((e = cudaMemcpy(c->d_sp, t.sp.data(), n * sizeof(u32), cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e, "upload");
    if ((e = cudaMemcpy(c->d_rcp, t.rcp.data(), n * sizeof(u64), cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e, "upload");
    if ((e = cudaMemcpy(c->d_inv, t.inv.data(), n * sizeof(u64), cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e, "upload");
    if (const char* cache = std::getenv("MPS_TUNE_CACHE")) mps_tune_load(c, cache);   // best effort
    *out = c;
    return MPS_OK;
}

int mps_close(mps_ctx* c) {
    if (!c) return MPS_E_ARG;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (WaveSlot& w : c->slot) slot_free(w);
    for (void* p : {(void*)c->d_sp, (void*)c->d_rcp, (void*)c->d_inv, (void*)c->d_ctr, (void*)c->d_surv,
                    (void*)c->d_surv_item, (void*)c->d_ent, (void*)c->d_rel, (void*)c->d_items, (void*)c->d_state})
        if (p) cudaFree(p);
    if (c->h_ctr) cudaFreeHost(c->h_ctr);
    if (c->h_rel) cudaFreeHost(c->h_rel);
    for (cudaEvent_t ev : {c->ev0, c->ev1, c->evb0, c->evb1})
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : c->evk)
        if (ev) cudaEventDestroy(ev);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return MPS_OK;
}

const char* mps_last_error(const mps_ctx* c) { return c ? c->err.c_str() : "no context"; }

int mps_get_stats(const mps_ctx* c, mps_stats* out) {
    if (!c || !out) return MPS_E_ARG;
    *out = c->stats;
    return MPS_OK;
}

int mps_chunk_relations(mps_ctx* c, uint64_t lo, uint64_t hi, const mps_item* item, mps_relation* out, size_t cap,
                        size_t* n_out) {
    if (int r = check_ctx(c)) return r;
    if (!out && cap) return fail(c, MPS_E_ARG, "out is NULL");
    begin_call(c);
    std::vector<RawRelation> rel;
    if (int r = relations_of(c, item, lo, hi, rel)) return r;
    if (int r = end_call(c)) return r;
    sort_by_p(rel);
    return copy_out(c, rel, out, nullptr, cap, n_out);
}

int mps_item_relations(mps_ctx* c, const mps_item* item, mps_relation* out, size_t cap, size_t* n_out) {
    if (!item) return fail(c, MPS_E_ARG, "item is NULL");
    if (c && c->tun.plain) return mps_chunk_relations(c, item->P0, item->P1, item, out, cap, n_out);
    if (int r = check_ctx(c)) return r;
    DevItem d;
    LaunchCfg g;
    if (int r = make_dev_item(c, item, 0, &d, &g)) return r;
    begin_call(c);
    std::vector<RawRelation> rel;
    c->item_K.assign(1, d.K);
    c->item_cfg.assign(1, g);
    if (int r = upload_items(c, &d, 1)) return r;
    if (int r = run_waves(c, {item->P0}, {item->P1}, rel)) return r;
    if (int r = end_call(c)) return r;
    sort_by_p(rel);
    return copy_out(c, rel, out, nullptr, cap, n_out);
}

int mps_sieve_filter(mps_ctx* c, uint64_t lo, uint64_t hi, const mps_item* item, uint64_t* out, size_t cap,
                     size_t* n_out) {
    if (int r = check_ctx(c)) return r;
    if (!(hi < kTwo62 && lo > 3)) return fail(c, MPS_E_RANGE, "the GPU sieve takes 3 < lo and hi < 2^62");
    begin_call(c);
    std::vector<RawRelation> rel;
    if (int r = relations_of(c, item, lo, hi, rel)) return r;
    if (int r = end_call(c)) return r;
    sort_by_p(rel);
    if (n_out) *n_out = rel.size();
    c->stats.relations = rel.size();
    if (rel.size() > cap) return fail(c, MPS_E_CAPACITY, "output buffer too small");
    for (size_t i = 0; i < rel.size(); ++i) out[i] = rel[i].p;
    return MPS_OK;
}

int mps_filter(mps_ctx* c, const uint64_t* primes, size_t n, const mps_item* item, uint8_t* flags) {
    if (int r = check_ctx(c)) return r;
    if (n == 0) return MPS_OK;
    if (!primes || !flags) return fail(c, MPS_E_ARG, "NULL buffer");
    DevItem d;
    LaunchCfg g;
    if (int r = make_dev_item(c, item, 0, &d, &g)) return r;
    for (size_t i = 0; i < n; ++i)
        if (primes[i] >= kTwo62) return fail(c, MPS_E_RANGE, "primes must be below 2^62");
    begin_call(c);
    if (int r = upload_items(c, &d, 1)) return r;
    const u64 chunk = c->tun.chunk_odds;
    std::vector<RawRelation> rel;
    for (size_t off = 0; off < n; off += chunk) {
        const u64 cnt = std::min<u64>(chunk, n - off);
        if (int r = ensure(c, &c->d_surv, &c->surv_cap, std::max<u64>(cnt + 16, chunk + 16), "survivor buffer")) return r;
        if (int r = ensure(c, &c->d_ent, &c->ent_cap, std::max<u64>(cnt, 1 << 16), "entry buffer")) return r;
        if (int r = ensure_rel(c, std::max<u64>(c->rel_cap, 1 << 18))) return r;
        u32 tbits, mb;
        table_for(c, g, d.K, &tbits, &mb);
        const u32 warps = g.warps;
        int bgrid = 0;
        if (int r = bsgs_grid(c, tbits, warps, g.kind, &bgrid)) return r;
        cudaStream_t s = c->stream;
        CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(Counters), s), "counter reset");
        CK(cudaMemcpyAsync(c->d_surv, primes + off, cnt * sizeof(u64), cudaMemcpyHostToDevice, s), "prime upload");
        Counters h{};
        h.survivors = cnt;
        CK(cudaMemcpyAsync(&c->d_ctr->survivors, &h.survivors, sizeof(u64), cudaMemcpyHostToDevice, s), "count upload");
        PrepArgs pa{};
        pa.surv = c->d_surv; pa.surv_cap = c->surv_cap; pa.item0 = 0; pa.items = c->d_items;
        pa.ent = c->d_ent; pa.ent_cap = c->ent_cap; pa.rel = c->d_rel; pa.rel_cap = c->rel_cap; pa.full_mr = c->tun.full_mr;
        pa.m_cap = launch_m_cap(c, g, tbits);
        pa.m_round = g.lanes * g.chains;
        BsgsArgs ba{};
        ba.ent = c->d_ent; ba.ent_cap = c->ent_cap; ba.rel = c->d_rel; ba.rel_cap = c->rel_cap;
        ba.tbits = tbits; ba.warps_per_block = warps; ba.persistent = 1; ba.chains = g.chains; ba.table_kind = g.kind;
        ba.load_shift = g.load_shift;
        ba.fill = g.fill;
        ba.lanes = for_range(g, *std::max_element(primes + off, primes + off + cnt) + 1).lanes;
        ba.max_p = *std::max_element(primes + off, primes + off + cnt);
        OrderArgs oa{};
        oa.rel = c->d_rel; oa.rel_cap = c->rel_cap; oa.items = c->d_items; oa.tables = c->tables();
        CK(launch_prep(pa, c->d_ctr, grid_for(c, 16), s), "prep launch");
        CK(launch_bsgs(ba, c->d_ctr, bgrid, s), "bsgs launch");
        CK(launch_order(oa, c->d_ctr, grid_for(c, 4), s), "order launch");
        CK(cudaMemcpyAsync(c->h_ctr, c->d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s), "count read");
        CK(cudaStreamSynchronize(s), "filter");
        if (c->h_ctr->status & (kStatusEntryOverflow | kStatusRelationOverflow | kStatusOrderFailed | kStatusBadLaunch))
            return fail(c, MPS_E_CUDA, "filter buffers overflowed");
        const u64 nr = c->h_ctr->relations;
        if (nr) {
            CK(cudaMemcpy(c->h_rel, c->d_rel, nr * sizeof(RawRelation), cudaMemcpyDeviceToHost), "relation read");
            for (u64 i = 0; i < nr; ++i)
                if (c->h_rel[i].q != ~0ull) rel.push_back(c->h_rel[i]);
        }
        c->stats.kernel_launches += 3;
    }
    if (int r = end_call(c)) return r;
    // flags by p (host-supplied primes may repeat or be unsorted)
    std::vector<u64> ps;
    ps.reserve(rel.size());
    for (const RawRelation& r : rel) ps.push_back(r.p);
    std::sort(ps.begin(), ps.end());
    for (size_t i = 0; i < n; ++i) flags[i] = std::binary_search(ps.begin(), ps.end(), primes[i]) ? 1 : 0;
    c->stats.relations = rel.size();
    return MPS_OK;
}

int mps_batch_relations(mps_ctx* c, const mps_item* items, size_t n_items, mps_relation* out, uint32_t* out_item,
                        size_t cap, size_t* n_out) {
    if (int r = check_ctx(c)) return r;
    if (!items && n_items) return fail(c, MPS_E_ARG, "items is NULL");
    std::vector<DevItem> d(n_items);
    std::vector<LaunchCfg> cfg(n_items);
    for (size_t i = 0; i < n_items; ++i)
        if (int r = make_dev_item(c, &items[i], (u32)i, &d[i], &cfg[i])) return r;
    begin_call(c);
    std::vector<RawRelation> rel;
    c->item_K.assign(n_items, 0);
    for (size_t i = 0; i < n_items; ++i) c->item_K[i] = d[i].K;
    c->item_cfg = cfg;
    if (int r = upload_items(c, d.data(), n_items)) return r;
    if (c->tun.plain) {
        // the plain path: one item after another, one chunk at a time
        for (size_t i = 0; i < n_items; ++i)
            if (int r = run_range(c, items[i].P0, items[i].P1, (u32)i, d[i].K, cfg[i], rel)) return r;
    } else {
        std::vector<u64> lo(n_items), hi(n_items);
        for (size_t i = 0; i < n_items; ++i) {
            lo[i] = items[i].P0;
            hi[i] = items[i].P1;
        }
        if (int r = run_waves(c, lo, hi, rel)) return r;
    }
    if (int r = end_call(c)) return r;
    sort_by_p(rel);
    return copy_out(c, rel, out, out_item, cap, n_out);
}

int mps_take_relations(mps_ctx* c, mps_relation* out, uint32_t* out_item, size_t cap, size_t* n_out) {
    if (!c) return MPS_E_ARG;
    if (!out && cap) return fail(c, MPS_E_ARG, "out is NULL");
    return copy_out(c, c->last, out, out_item, cap, n_out);
}


int mps_serve_config_default(mps_serve_config* cfg) {
    if (!cfg) return MPS_E_ARG;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->struct_size = sizeof(mps_serve_config);
    cfg->max_active = 256;
    cfg->mem_budget_bytes = 4ull << 30;
    cfg->piece_odds = 1ull << 22;
    return MPS_OK;
}

int mps_serve_open(int device, const mps_tuning* tuning, const mps_serve_config* cfg, mps_server** out) {
    if (!out) return MPS_E_ARG;
    *out = nullptr;
    mps_serve_config conf;
    mps_serve_config_default(&conf);
    if (cfg) {
        if (cfg->struct_size != sizeof(mps_serve_config)) return MPS_E_ARG;
        if (cfg->max_active) conf.max_active = cfg->max_active;
        if (cfg->mem_budget_bytes) conf.mem_budget_bytes = cfg->mem_budget_bytes;
        if (cfg->piece_odds) conf.piece_odds = cfg->piece_odds;
    }
    conf.max_active = std::min<u32>(conf.max_active, kMaxRuns);
    mps_ctx* c = nullptr;
    if (int r = mps_open(device, tuning, &c)) return r;
    if (int r = reserve_items(c, conf.max_active)) {
        mps_close(c);
        return r;
    }
    c->item_K.assign(conf.max_active, 0);
    c->item_cfg.assign(conf.max_active, default_cfg(c));
    for (WaveSlot& w : c->slot)
        if (int r = slot_alloc(c, w)) {
            mps_close(c);
            return r;
        }
    c->slots_ready = true;
    // the reservation pool: the budget, at most 90% of the device memory still free
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        mps_close(c);
        return MPS_E_CUDA;
    }
    const u64 pool_bytes = std::min<u64>(conf.mem_budget_bytes, (u64)(0.9 * (double)free_b)) & ~255ull;
    unsigned char* pool = nullptr;
    if (pool_bytes < 4096 || cudaMalloc((void**)&pool, pool_bytes) != cudaSuccess) {
        mps_close(c);
        return MPS_E_CUDA;
    }
    mps_server* sv = new mps_server();
    sv->ctx = c;
    sv->pool = pool;
    sv->alloc.reset(pool_bytes);
    sv->cfg = conf;
    sv->slot_owner.assign(conf.max_active, 0);
    sv->worker = std::thread(serve_loop, sv);
    *out = sv;
    return MPS_OK;
}

int mps_serve_submit(mps_server* sv, const mps_item* item, uint64_t* ticket) {
    if (!sv || !item || !ticket) return MPS_E_ARG;
    ServeReq q;
    if (int r = make_dev_item(sv->ctx, item, 0, &q.d)) return r;
    std::lock_guard<std::mutex> g(sv->mu);
    if (sv->fatal) return MPS_E_STATE;
    if (sv->stop) return MPS_E_STATE;
    q.ticket = sv->next_ticket++;
    q.item = *item;
    q.mem = expected_relations(q.d, *item) * sizeof(RawRelation);
    q.t_submit = std::chrono::steady_clock::now();
    *ticket = q.ticket;
    sv->reqs[q.ticket] = std::move(q);
    sv->queue.push_back(*ticket);
    sv->cv_work.notify_one();
    return MPS_OK;
}

int mps_serve_wait(mps_server* sv, uint64_t ticket, double timeout_s, mps_serve_status* st) {
    if (!sv) return MPS_E_ARG;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return MPS_E_ARG;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(std::max(0.0, timeout_s));
    while (it->second.state < 2) {
        if (sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && it->second.state < 2) break;
    }
    const ServeReq& q = it->second;
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->ticket = q.ticket;
        st->state = q.state;
        st->error = q.error;
        st->relations = q.rel.size();
        st->p_done = q.cursor;
        st->reserved_bytes = q.mem;
        st->relations_on_device = q.relations_on_device ? 1 : 0;
        if (q.state >= 2) {
            st->latency_ms = ms_between(q.t_submit, q.t_done);
            st->queue_ms = q.slot >= 0 || q.state == 2 ? ms_between(q.t_submit, q.t_admit) : 0.0;
        }
    }
    if (q.state == 3) return q.error ? q.error : MPS_E_CUDA;
    return q.state == 2 ? MPS_OK : MPS_E_TIMEOUT;
}

int mps_serve_result(mps_server* sv, uint64_t ticket, mps_relation* out, size_t cap, size_t* n_out) {
    if (!sv) return MPS_E_ARG;
    std::lock_guard<std::mutex> g(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return MPS_E_ARG;
    const ServeReq& q = it->second;
    if (q.state != 2) return q.state == 3 ? MPS_E_STATE : MPS_E_TIMEOUT;
    if (n_out) *n_out = q.rel.size();
    if (q.rel.size() > cap) return MPS_E_CAPACITY;
    for (size_t i = 0; i < q.rel.size(); ++i) {
        out[i].p = q.rel[i].p;
        out[i].M = q.rel[i].M;
        out[i].q = q.rel[i].q;
    }
    return MPS_OK;
}

int mps_serve_release(mps_server* sv, uint64_t ticket) {
    if (!sv) return MPS_E_ARG;
    std::lock_guard<std::mutex> g(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return MPS_E_ARG;
    if (it->second.state < 2) return MPS_E_STATE;
    sv->reqs.erase(it);
    return MPS_OK;
}

int mps_serve_pool(mps_server* sv, uint64_t* pool_bytes, uint64_t* reserved_bytes, uint32_t* active, uint32_t* queued) {
    if (!sv) return MPS_E_ARG;
    std::lock_guard<std::mutex> g(sv->mu);
    if (pool_bytes) *pool_bytes = sv->alloc.total();
    if (reserved_bytes) *reserved_bytes = sv->alloc.used();
    if (active) *active = sv->active;
    if (queued) *queued = (uint32_t)sv->queue.size();
    return MPS_OK;
}

int mps_serve_checkpoint(mps_server* sv, uint64_t ticket, uint64_t* p_done, uint64_t* n_rel) {
    if (!sv) return MPS_E_ARG;
    // The device table holds, per item, the highest P of any committed wave
    // and the relations committed; pieces are issued in increasing P, so
    // every P below min(that, the lowest piece still in flight, the next
    // piece to issue) is sieved.
    int slot = -1;
    u64 cursor = 0, nr = 0, limit = 0, P0 = 0;
    int state = 0;
    {
        std::lock_guard<std::mutex> g(sv->mu);
        auto it = sv->reqs.find(ticket);
        if (it == sv->reqs.end()) return MPS_E_ARG;
        const ServeReq& q = it->second;
        slot = q.slot;
        state = q.state;
        cursor = q.state == 2 ? q.item.P1 : q.item.P0;
        nr = q.rel.size();
        limit = q.piece_lo.empty() ? q.cursor : *q.piece_lo.begin();
        P0 = q.item.P0;
    }
    if (state == 1 && slot >= 0) {
        ItemState h{};
        cudaSetDevice(sv->ctx->device);
        if (cudaMemcpy(&h, sv->ctx->d_state + slot, sizeof(ItemState), cudaMemcpyDeviceToHost) != cudaSuccess)
            return MPS_E_CUDA;
        cursor = std::max<u64>(P0, std::min<u64>(h.p_done, limit));
        nr = h.n_rel;
    }
    if (p_done) *p_done = cursor;
    if (n_rel) *n_rel = nr;
    return MPS_OK;
}

int mps_serve_close(mps_server* sv) {
    if (!sv) return MPS_E_ARG;
    {
        std::lock_guard<std::mutex> g(sv->mu);
        sv->stop = true;
        sv->cv_work.notify_all();
    }
    if (sv->worker.joinable()) sv->worker.join();
    if (sv->pool) {
        cudaSetDevice(sv->ctx->device);
        cudaFree(sv->pool);
    }
    mps_close(sv->ctx);
    delete sv;
    return MPS_OK;
}

int mps_count_primes(mps_ctx* c, uint64_t lo, uint64_t hi, uint64_t* count) {
    if (int r = check_ctx(c)) return r;
    if (!count) return fail(c, MPS_E_ARG, "count is NULL");
    if (hi > kTwo62) return fail(c, MPS_E_RANGE, "hi must not exceed 2^62");
    *count = 0;
    const u64 chunk = c->tun.chunk_odds;
    for (u64 a = lo; a < hi;) {
        const u64 lo_odd = std::max<u64>(a, 3) | 1ull;
        u64 b = hi;
        if (lo_odd < hi && (hi - lo_odd + 1) / 2 > chunk) b = lo_odd + 2 * chunk;
        const u64 n_odds = lo_odd < b ? (b - lo_odd + 1) / 2 : 0;
        if (int r = ensure(c, &c->d_surv, &c->surv_cap, chunk + 16, "survivor buffer")) return r;
        SieveArgs sa{};
        sa.lo_odd = lo_odd; sa.n_odds = n_odds; sa.hi = b; sa.include_two = (a <= 2 && b > 2);
        sa.n_primes = sieve_prime_count(b);
        CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(Counters), c->stream), "counter reset");
        CK(launch_sieve(sa, c->tables(), c->d_surv, nullptr, c->surv_cap, c->d_ctr, c->stream), "sieve launch");
        CK(launch_count_primes(c->d_surv, c->surv_cap, c->d_ctr, grid_for(c, 8), c->stream), "count launch");
        CK(cudaMemcpyAsync(c->h_ctr, c->d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, c->stream), "count read");
        CK(cudaStreamSynchronize(c->stream), "count");
        if (c->h_ctr->status) return fail(c, MPS_E_CUDA, "survivor buffer overflow while counting");
        *count += c->h_ctr->primes;
        a = b;
    }
    return MPS_OK;
}

int mps_measure_peaks(mps_ctx* c, double* fmul_per_s, double* mmul_per_s, double* imad_per_s) {
    if (int r = check_ctx(c)) return r;
    u64* sink = nullptr;
    CK(cudaMalloc((void**)&sink, 64), "alloc");
    const int grid = c->num_sms * 8;
    const u32 iters = 4096;
    float ms[3] = {0, 0, 0};
    cudaError_t e = cudaSuccess;
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {     // the second repetition is kept
        for (int k = 0; k < 3 && e == cudaSuccess; ++k) {
            e = cudaEventRecord(c->ev0, c->stream);
            if (e != cudaSuccess) break;
            if (k == 0) e = launch_fmul_peak(0x00005639F00D1ull, iters, grid, sink, c->stream);
            if (k == 1) e = launch_mmul_peak(0x00005639F00D1ull, iters, grid, sink, c->stream);
            if (k == 2) e = launch_imad_peak(iters * 8, grid, (u32*)sink, c->stream);
            if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(c->ev1);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms[k], c->ev0, c->ev1);
        }
    }
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_fail(c, e, "peak probes");
    const double ops = (double)grid * 256.0 * 8.0 * iters;
    if (fmul_per_s) *fmul_per_s = ops / (ms[0] * 1e-3);
    if (mmul_per_s) *mmul_per_s = ops / (ms[1] * 1e-3);
    if (imad_per_s) *imad_per_s = ops * 8.0 / (ms[2] * 1e-3);
    return MPS_OK;
}

int mps_autotune(mps_ctx* c, const mps_item* items, size_t n_items, mps_tune_report* out, size_t cap,
                 size_t* n_out) {
    if (int r = check_ctx(c)) return r;
    if (!items && n_items) return fail(c, MPS_E_ARG, "items is NULL");
    if (!out && cap) return fail(c, MPS_E_ARG, "out is NULL");
    constexpr u64 kCalibSpan = 1ull << 25;
    const LaunchCfg base = default_cfg(c);
    std::vector<LaunchCfg> cands{base};
    for (u32 kind : {0u, 3u})
        for (u32 ch : {1u, 2u, 4u})
            for (u32 w : {4u, 8u}) {
                LaunchCfg g;
                g.kind = kind;
                g.chains = ch;
                g.warps = w;
                if (g != base) cands.push_back(g);
            }
    // lanes per prime: groups of 16 or 8 lanes (table kind 2, 1 or 2 chains)
    for (u32 lanes : {16u, 8u})
        for (u32 ch : {1u, 2u})
            for (u32 w : {4u, 8u}) {
                LaunchCfg g;
                g.kind = 2;
                g.load_shift = 2;
                g.chains = ch;
                g.warps = w;
                g.lanes = lanes;
                cands.push_back(g);
            }
    std::vector<mps_tune_report> reps;
    std::set<u64> seen;
    for (size_t i = 0; i < n_items; ++i) {
        DevItem d;
        const char* why = "";
        if (int r = item_constants(&items[i], c->tun.class_modulus, 0, &d, &why)) return fail(c, r, why);
        const u64 key = tune_key(d.K, d.cm, items[i].P0);
        if (!seen.insert(key).second || !d.has_work) continue;
        const u64 lo = items[i].P0, hi = std::min<u64>(items[i].P1, items[i].P0 + kCalibSpan);
        double best_ms = 0, base_ms = 0, sieve_base_ms = 0, sieve_best_ms = 0;
        u64 entries = 0;
        LaunchCfg best = base;
        std::vector<RawRelation> first;
        // phase 1: the BSGS configuration by the BSGS kernel's time; phase 2: with
        // it, the table fill and the baby-step scale (fingerprint words only);
        // phase 3: the sieve's segment size by the sieve kernel's time
        constexpr u32 kFills[] = {224u, 192u, 160u, 128u};
        constexpr u32 kScales[] = {224u, 192u, 160u, 128u};
        const size_t n_bsgs = cands.size();
        const size_t n_fill = n_bsgs + (sizeof(kFills) / sizeof(kFills[0])) * (sizeof(kScales) / sizeof(kScales[0]));
        const size_t n_all = n_fill + 3;
        size_t timed = 0;
        for (size_t k = 0; k < n_all; ++k) {
            LaunchCfg g;
            if (k < n_bsgs) {
                g = cands[k];
            } else if (k < n_fill) {                            // phase 2 keeps the chosen BSGS settings
                if (best.kind != 0 && best.kind != 3) continue;
                const size_t f = (k - n_bsgs) / (sizeof(kScales) / sizeof(kScales[0]));
                const size_t sc = (k - n_bsgs) % (sizeof(kScales) / sizeof(kScales[0]));
                g = best;
                g.fill = kFills[f];
                g.scale = kScales[sc];
                if (g == best) continue;
            } else {                                            // phase 3 keeps the chosen BSGS settings
                g = best;
                g.seg_words = 1024u << (k - n_fill);
            }
            if (g.lanes != 32 && hi > kFp64Limit) continue;    // groups run the FP64 solve only
            u32 tb, mb;
            table_for(c, g, d.K, &tb, &mb);
            d.max_baby = mb;
            d.baby_scale = g.scale;
            if (bsgs_smem_bytes(tb, g.warps, g.kind) > c->smem_optin) continue;
            if (int r = upload_items(c, &d, 1)) return r;
            ++timed;
            double ms = 0, sms = 0;
            for (int rep = 0; rep < 2; ++rep) {                 // the second run is timed
                std::vector<RawRelation> rel;
                std::memset(&c->stats, 0, sizeof(c->stats));
                if (int r = run_chunk(c, lo, hi, 0, d.K, g, rel)) return r;
                ms = c->stats.bsgs_ms;
                sms = c->stats.sieve_ms;
                entries = c->stats.entries;
                sort_by_p(rel);
                if (k == 0 && rep == 0) {
                    first = rel;
                } else if (rel.size() != first.size() ||
                           !std::equal(rel.begin(), rel.end(), first.begin(), [](const RawRelation& a, const RawRelation& b) {
                               return a.p == b.p && a.M == b.M && a.q == b.q;
                           })) {
                    return fail(c, MPS_E_CUDA, "tuning candidates gave different relations");
                }
            }
            if (k < n_fill) {
                if (k == 0) base_ms = ms;
                if (k == 0 || ms < best_ms) {
                    best_ms = ms;
                    best = g;
                }
            } else {
                if (g.seg_words == base.seg_words) sieve_base_ms = sms;
                if (k == n_fill || sms < sieve_best_ms) {
                    sieve_best_ms = sms;
                    best.seg_words = g.seg_words;
                }
            }
        }
        const double per = entries ? 1e6 / (double)entries : 0.0;
        TuneEntry te;
        te.cfg = best;
        te.ns_per_prime = best_ms * per;
        c->tuned[key] = te;
        mps_tune_report rp{};
        rp.k_bits = (u32)(key >> 40);
        rp.mod = (u32)((key >> 8) & 4095);
        rp.p_digits = (u32)(key & 255);
        rp.candidates = (u32)timed;
        rp.table_kind = best.kind;
        rp.load_shift = best.load_shift;
        rp.chains = best.chains;
        rp.warps = best.warps;
        rp.seg_words = best.seg_words;
        rp.lanes = best.lanes;
        rp.table_fill = best.fill;
        rp.baby_scale = best.scale;
        rp.sieve_best_ms = sieve_best_ms;
        rp.sieve_default_ms = sieve_base_ms;
        rp.best_ns_per_prime = best_ms * per;
        rp.default_ns_per_prime = base_ms * per;
        rp.calib_bsgs_primes = entries;
        reps.push_back(rp);
    }
    std::memset(&c->stats, 0, sizeof(c->stats));
    if (n_out) *n_out = reps.size();
    if (reps.size() > cap) return fail(c, MPS_E_CAPACITY, "report buffer too small");
    for (size_t k = 0; k < reps.size(); ++k) out[k] = reps[k];
    return MPS_OK;
}

int mps_tune_save(const mps_ctx* c, const char* path) {
    if (!c || !path) return MPS_E_ARG;
    FILE* f = std::fopen(path, "w");
    if (!f) return MPS_E_ARG;
    std::fprintf(f, "mps-tune 4\n");
    for (const auto& kv : c->tuned)
        std::fprintf(f, "%llu %u %u %u %u %u %u %u %u %.3f\n", (unsigned long long)kv.first, kv.second.cfg.kind,
                     kv.second.cfg.load_shift, kv.second.cfg.chains, kv.second.cfg.warps, kv.second.cfg.seg_words,
                     kv.second.cfg.lanes, kv.second.cfg.fill, kv.second.cfg.scale, kv.second.ns_per_prime);
    return std::fclose(f) == 0 ? MPS_OK : MPS_E_ARG;
}

int mps_tune_load(mps_ctx* c, const char* path) {
    if (!c || !path) return MPS_E_ARG;
    FILE* f = std::fopen(path, "r");
    if (!f) return fail(c, MPS_E_ARG, std::string("cannot open ") + path);
    char head[32] = {0};
    if (!std::fgets(head, sizeof(head), f) || std::strncmp(head, "mps-tune 4", 10) != 0) {
        std::fclose(f);
        return fail(c, MPS_E_ARG, "not a tuning file");
    }
    unsigned long long key;
    unsigned kind, ls, ch, w, sw, lanes, fill, scale;
    double ns;
    while (std::fscanf(f, "%llu %u %u %u %u %u %u %u %u %lf", &key, &kind, &ls, &ch, &w, &sw, &lanes, &fill, &scale,
                       &ns) == 10) {
        // only configurations the kernels are built for
        if (kind > 3 || ls < 1 || ls > 4 || (ch != 1 && ch != 2 && ch != 4) || w < 1 || w > 8 ||
            (sw != 1024 && sw != 2048 && sw != 4096) || (lanes != 32 && lanes != 16 && lanes != 8) ||
            (lanes != 32 && (kind != 2 || ch == 4)) || fill < 1 || fill > 256 || scale < 1 || scale > 1024)
            continue;
        TuneEntry te;
        te.cfg.kind = kind;
        te.cfg.load_shift = ls;
        te.cfg.chains = ch;
        te.cfg.warps = w;
        te.cfg.seg_words = sw;
        te.cfg.lanes = lanes;
        te.cfg.fill = fill;
        te.cfg.scale = scale;
        te.ns_per_prime = ns;
        c->tuned[key] = te;
    }
    std::fclose(f);
    return MPS_OK;
}

int mps_tune_clear(mps_ctx* c) {
    if (!c) return MPS_E_ARG;
    c->tuned.clear();
    return MPS_OK;
}

int mps_measure_smem_peak(mps_ctx* c, double* atomic_or_per_s) {
    if (int r = check_ctx(c)) return r;
    if (!atomic_or_per_s) return fail(c, MPS_E_ARG, "NULL output");
    u32* sink = nullptr;
    CK(cudaMalloc((void**)&sink, 64), "alloc");
    const int grid = c->num_sms * 8;
    const u32 iters = 2048;
    float ms = 0;
    cudaError_t e = cudaSuccess;
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {     // the second repetition is kept
        e = cudaEventRecord(c->ev0, c->stream);
        if (e == cudaSuccess) e = launch_smem_or_peak(iters, grid, sink, c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(c->ev1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    }
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_fail(c, e, "shared-memory probe");
    *atomic_or_per_s = (double)grid * 256.0 * 8.0 * iters / (ms * 1e-3);
    return MPS_OK;
}

int mps_test_survivors(mps_ctx* c, uint64_t lo, uint64_t hi, uint64_t* out, size_t cap, size_t* n_out) {
    if (int r = check_ctx(c)) return r;
    if (hi > kTwo62 || lo >= hi) return fail(c, MPS_E_RANGE, "need lo < hi <= 2^62");
    const u64 lo_odd = std::max<u64>(lo, 3) | 1ull;
    const u64 n_odds = lo_odd < hi ? (hi - lo_odd + 1) / 2 : 0;
    if (n_odds > (1ull << 30)) return fail(c, MPS_E_RANGE, "range too wide for the test hook");
    if (int r = ensure(c, &c->d_surv, &c->surv_cap, std::max<u64>(n_odds + 16, c->surv_cap), "survivor buffer")) return r;
    SieveArgs sa{};
    sa.lo_odd = lo_odd; sa.n_odds = n_odds; sa.hi = hi; sa.include_two = 0;
    sa.n_primes = sieve_prime_count(hi);
    CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(Counters), c->stream), "counter reset");
    CK(launch_sieve(sa, c->tables(), c->d_surv, nullptr, c->surv_cap, c->d_ctr, c->stream), "sieve launch");
    CK(cudaMemcpyAsync(c->h_ctr, c->d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, c->stream), "count read");
    CK(cudaStreamSynchronize(c->stream), "sieve");
    const u64 ns = c->h_ctr->survivors;
    if (n_out) *n_out = ns;
    if (ns > cap) return fail(c, MPS_E_CAPACITY, "output buffer too small");
    CK(cudaMemcpy(out, c->d_surv, ns * sizeof(u64), cudaMemcpyDeviceToHost), "survivor read");
    std::sort(out, out + ns);
    return MPS_OK;
}

int mps_test_is_prime(mps_ctx* c, const uint64_t* n, size_t count, uint8_t* out) {
    if (int r = check_ctx(c)) return r;
    for (size_t i = 0; i < count; ++i)
        if (n[i] >= kTwo62) return fail(c, MPS_E_RANGE, "n must be below 2^62");
    u64* dn = nullptr;
    u32* dout = nullptr;
    CK(cudaMalloc((void**)&dn, std::max<size_t>(count, 1) * sizeof(u64)), "alloc");
    CK(cudaMalloc((void**)&dout, std::max<size_t>(count, 1) * sizeof(u32)), "alloc");
    std::vector<u32> h(count);
    cudaError_t e = cudaMemcpy(dn, n, count * sizeof(u64), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_is_prime(dn, dout, count, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), dout, count * sizeof(u32), cudaMemcpyDeviceToHost);
    cudaFree(dn);
    cudaFree(dout);
    if (e != cudaSuccess) return cuda_fail(c, e, "is_prime test");
    for (size_t i = 0; i < count; ++i) out[i] = (uint8_t)h[i];
    return MPS_OK;
}

int mps_test_bsgs(mps_ctx* c, const uint64_t* cases, size_t count, uint32_t table_bits, uint64_t* j_out) {
    if (int r = check_ctx(c)) return r;
    if (table_bits < 5 || table_bits > 14) return fail(c, MPS_E_ARG, "table_bits must be in [5, 14]");
    for (size_t i = 0; i < count; ++i) {
        const uint64_t* k = cases + 5 * i;
        if (k[0] < 3 || !(k[0] & 1) || k[0] >= kTwo62) return fail(c, MPS_E_RANGE, "p must be odd, 3 <= p < 2^62");
        if (k[1] == 0 || k[1] >= k[0] || k[2] == 0 || k[2] >= k[0] || k[3] == 0 || k[3] >= k[0])
            return fail(c, MPS_E_ARG, "B, G0, t must lie in [1, p)");
    }
    u64* dc = nullptr;
    u64* dj = nullptr;
    CK(cudaMalloc((void**)&dc, std::max<size_t>(count, 1) * 5 * sizeof(u64)), "alloc");
    CK(cudaMalloc((void**)&dj, std::max<size_t>(count, 1) * sizeof(u64)), "alloc");
    std::memset(&c->stats, 0, sizeof(c->stats));
    cudaError_t e = cudaMemcpy(dc, cases, count * 5 * sizeof(u64), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaEventRecord(c->evb0, c->stream);
    if (e == cudaSuccess) e = launch_bsgs_direct(dc, dj, count, table_bits, c->tun.table_kind, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->evb1, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, c->evb0, c->evb1);
    c->stats.bsgs_ms = ms;
    c->stats.bsgs_launches = 1;
    c->stats.kernel_launches = 1;
    if (e == cudaSuccess) e = cudaMemcpy(j_out, dj, count * sizeof(u64), cudaMemcpyDeviceToHost);
    cudaFree(dc);
    cudaFree(dj);
    if (e != cudaSuccess) return cuda_fail(c, e, "bsgs test");
    return MPS_OK;
}

int mps_test_order(mps_ctx* c, const uint64_t* bp, size_t count, uint64_t* q_out) {
    if (int r = check_ctx(c)) return r;
    for (size_t i = 0; i < count; ++i) {
        const u64 b = bp[2 * i], p = bp[2 * i + 1];
        if (p < 3 || p >= kTwo62 || b % p == 0) return fail(c, MPS_E_ARG, "need 3 <= p < 2^62 and p not dividing b");
    }
    u64* db = nullptr;
    u64* dq = nullptr;
    CK(cudaMalloc((void**)&db, std::max<size_t>(count, 1) * 2 * sizeof(u64)), "alloc");
    CK(cudaMalloc((void**)&dq, std::max<size_t>(count, 1) * sizeof(u64)), "alloc");
    cudaError_t e = cudaMemcpy(db, bp, count * 2 * sizeof(u64), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_order_direct(db, dq, count, c->tables(), c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(q_out, dq, count * sizeof(u64), cudaMemcpyDeviceToHost);
    cudaFree(db);
    cudaFree(dq);
    if (e != cudaSuccess) return cuda_fail(c, e, "order test");
    return MPS_OK;
}

}  // extern "C"
