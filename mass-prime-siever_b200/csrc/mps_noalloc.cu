// mps_noalloc.cu -- relations of one small prime range with no allocation.
//
// Who needs this: a caller that must not allocate device memory at the point
// where it sieves.  Examples: a host process whose device memory is owned by
// another framework's pool allocator (a raw cudaMalloc there fails once the
// pool has taken the memory, or fragments it), and a latency-bound loop that
// cannot afford cudaMalloc / cudaFree, which synchronise the whole device.
// The regular entry points (mps_open, mps_chunk_relations) allocate their
// buffers on first use and grow them on demand, so such callers cannot use
// them.
//
// Here all scratch memory -- counters, the item, the sieving-prime tables,
// survivors, BSGS entries, raw relations -- lives in ONE file-scope device
// array, g_noalloc_scratch, of kNoAllocBytes (8 MiB).  Every GPU that loads
// this library holds that array until the process exits.  Its address comes
// from cudaGetSymbolAddress, once per device, on the first call made on that
// device (with that device current); make the first call before capturing
// work on any stream into a CUDA graph.  Every call shares the one array and
// leaves the previous call's contents in it: the counters are cleared at the
// start of each pass.  Calls that overlap on the GPU (two host threads, or
// two devices' worth of work on one device at once) race on the array and
// must not be made.  No cudaMalloc, cudaFree, cudaMallocHost or other
// allocating routine is called, on the device or the host.
#include "../../include/mps_gpu.h"
#include "mps_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

using namespace mps;

namespace {

// Largest range one call takes: 2^19 integers (2^18 odd numbers).
constexpr u64 kNoAllocMaxSpan = 1ull << 19;
constexpr u64 kNoAllocOdds = kNoAllocMaxSpan / 2 + 2;
constexpr u64 kNoAllocEntries = 1ull << 16;
constexpr u64 kNoAllocRelations = 1ull << 14;
constexpr u32 kNoAllocMaxDevices = 64;

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffCounters = 0;
constexpr size_t kOffItem = align256(kOffCounters + sizeof(Counters));
constexpr size_t kOffSp = align256(kOffItem + sizeof(DevItem));
constexpr size_t kOffRcp = align256(kOffSp + kSievePrimes * sizeof(u32));
constexpr size_t kOffInv = align256(kOffRcp + kSievePrimes * sizeof(u64));
constexpr size_t kOffSurv = align256(kOffInv + kSievePrimes * sizeof(u64));
constexpr size_t kOffEnt = align256(kOffSurv + kNoAllocOdds * sizeof(u64));
constexpr size_t kOffRel = align256(kOffEnt + kNoAllocEntries * sizeof(Entry));
constexpr size_t kNoAllocUsed = align256(kOffRel + kNoAllocRelations * sizeof(RawRelation));
constexpr size_t kNoAllocBytes = 8u << 20;
static_assert(kNoAllocUsed <= kNoAllocBytes, "no-alloc scratch layout exceeds its array");

}  // namespace

// The scratch array (device memory reserved when the library is loaded).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_setup_lock;
unsigned char* g_scratch_dev[kNoAllocMaxDevices];   // device address per device, once known

// Host copies of the sieving-prime tables, built once in static storage.
u32 g_sp[kSievePrimes];
u64 g_rcp[kSievePrimes];
u64 g_inv[kSievePrimes];
bool g_tables_built = false;

void build_tables() {
    static bool comp[65536];
    u32 n = 0;
    for (u32 i = 3; i < 65536 && n < kSievePrimes; i += 2) {
        if (comp[i]) continue;
        g_sp[n] = i;
        g_rcp[n] = ~0ull / i;
        u64 x = i;
        for (int k = 0; k < 6; ++k) x *= 2 - i * x;
        g_inv[n] = x;
        ++n;
        for (u64 j = (u64)i * i; j < 65536; j += 2 * i) comp[j] = true;
    }
    g_tables_built = true;
}

// Address of the scratch array on the current device; sets it up (tables)
// on the first call for that device.  nullptr on failure.
unsigned char* scratch_for_current_device(int* code) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        *code = MPS_E_NODEV;
        return nullptr;
    }
    if (dev >= (int)kNoAllocMaxDevices) {
        *code = MPS_E_NODEV;
        return nullptr;
    }
    std::lock_guard<std::mutex> g(g_setup_lock);
    if (g_scratch_dev[dev]) return g_scratch_dev[dev];
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || ptr == nullptr) {
        *code = MPS_E_CUDA;
        return nullptr;
    }
    if (!g_tables_built) build_tables();
    unsigned char* base = (unsigned char*)ptr;
    if (cudaMemcpy(base + kOffSp, g_sp, sizeof(g_sp), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + kOffRcp, g_rcp, sizeof(g_rcp), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + kOffInv, g_inv, sizeof(g_inv), cudaMemcpyHostToDevice) != cudaSuccess) {
        *code = MPS_E_CUDA;
        return nullptr;
    }
    g_scratch_dev[dev] = base;
    return base;
}

u64 gcd_u64(u64 a, u64 b) {
    while (b) {
        const u64 t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// The item's device constants with the default tuning (same rules as the
// regular entry points: load_worktodo's checks plus P1 <= 2^62).
int item_constants(const mps_item* it, DevItem* d, u32* tbits) {
    if (!it) return MPS_E_ARG;
    if (it->P0 >= it->P1 || it->N0 >= it->N1) return MPS_E_ARG;
    if (it->P1 > (1ull << 62)) return MPS_E_RANGE;
    if ((unsigned __int128)((__int128)it->N1 - it->N0) > 10000000ull) return MPS_E_RANGE;
    const u64 cm = it->mod == 0 ? 1 : it->mod;
    if (it->res >= cm) return MPS_E_ARG;
    std::memset(d, 0, sizeof(*d));
    const __int128 b = (__int128)(((unsigned __int128)(u64)it->b_hi << 64) | it->b_lo);
    const __int128 c = (__int128)(((unsigned __int128)(u64)it->c_hi << 64) | it->c_lo);
    const unsigned __int128 babs = b < 0 ? (unsigned __int128)0 - (unsigned __int128)b : (unsigned __int128)b;
    const unsigned __int128 cabs = c < 0 ? (unsigned __int128)0 - (unsigned __int128)c : (unsigned __int128)c;
    d->babs_hi = (u64)(babs >> 64);
    d->babs_lo = (u64)babs;
    d->cabs_hi = (u64)(cabs >> 64);
    d->cabs_lo = (u64)cabs;
    d->b_neg = b < 0;
    d->c_neg = c < 0;
    d->N0_raw = it->N0;
    d->N1_raw = it->N1;
    d->N0 = it->N0 < 0 ? 0 : (u64)it->N0;
    d->N1 = it->N1 < 0 ? 0 : (u64)it->N1;
    d->cm = cm;
    d->n_start = d->N0 + ((it->res % cm) + cm - (d->N0 % cm)) % cm;
    d->has_work = (it->N1 > 0 && d->n_start < d->N1) ? 1 : 0;
    d->K = d->has_work ? (d->N1 - d->n_start + cm - 1) / cm : 0;
    const u64 l = cm / gcd_u64(cm, 5040) * 5040;
    const u64 Q = l <= 100800 ? l : 5040;
    d->Q = (u32)Q;
    d->Q_rcp = ~0ull / Q;
    d->cmQ = (u32)(cm % Q);
    d->nsQ = (u32)(d->n_start % Q);
    u64 x = Q;
    for (u64 f = 2; f * f <= x; ++f) {
        if (x % f) continue;
        d->qf_l[d->qf_n++] = (u32)f;
        while (x % f == 0) x /= f;
    }
    if (x > 1) d->qf_l[d->qf_n++] = (u32)x;
    const u64 m_opt = (u64)std::ceil(std::sqrt((double)std::max<u64>(d->K, 1)));
    u32 tb = 6;
    while ((1ull << tb) < 5 * m_opt && tb < 11) ++tb;
    *tbits = tb;
    d->max_baby = std::max<u32>((1u << tb) / 5, 1);
    return MPS_OK;
}

u32 prime_count_below_sqrt(u64 hi) {
    u32 n = 0;
    while (n < kSievePrimes && (u64)g_sp[n] * g_sp[n] < hi) ++n;
    return n;
}

// Host staging for one pass's raw relations (static storage, shared by calls).
RawRelation g_host_rel[kNoAllocRelations];

struct Sink {
    mps_relation* out;
    size_t cap;
    size_t n;
};

int run_pass(unsigned char* base, u64 lo, u64 hi, const DevItem& d, u32 tbits, int num_sms, Sink& sink) {
    Counters* ctr = (Counters*)(base + kOffCounters);
    DevItem* ditem = (DevItem*)(base + kOffItem);
    u64* surv = (u64*)(base + kOffSurv);
    Entry* ent = (Entry*)(base + kOffEnt);
    RawRelation* rel = (RawRelation*)(base + kOffRel);
    const SieveTables tables{(const u32*)(base + kOffSp), (const u64*)(base + kOffRcp), (const u64*)(base + kOffInv)};
    const cudaStream_t s = 0;

    const u64 lo_odd = std::max<u64>(lo, 3) | 1ull;
    SieveArgs sa{};
    sa.lo_odd = lo_odd;
    sa.n_odds = lo_odd < hi ? (hi - lo_odd + 1) / 2 : 0;
    sa.hi = hi;
    sa.include_two = (lo <= 2 && hi > 2) ? 1 : 0;
    sa.n_primes = prime_count_below_sqrt(hi);
    sa.item = 0;
    if (sa.n_odds == 0 && !sa.include_two) return MPS_OK;

    PrepArgs pa{};
    pa.surv = surv;
    pa.surv_cap = kNoAllocOdds;
    pa.item0 = 0;
    pa.items = ditem;
    pa.ent = ent;
    pa.ent_cap = kNoAllocEntries;
    pa.rel = rel;
    pa.rel_cap = kNoAllocRelations;
    BsgsArgs ba{};
    ba.ent = ent;
    ba.ent_cap = kNoAllocEntries;
    ba.rel = rel;
    ba.rel_cap = kNoAllocRelations;
    ba.tbits = tbits;
    ba.warps_per_block = 4;
    ba.persistent = 1;
    ba.chains = 2;
    ba.max_p = hi;
    OrderArgs oa{};
    oa.rel = rel;
    oa.rel_cap = kNoAllocRelations;
    oa.items = ditem;
    oa.tables = tables;

    const size_t smem = bsgs_smem_bytes(tbits, 4);
    const int bgrid = num_sms * std::max(1, std::min((int)(228 * 1024 / (smem + 1024)), 16));
    if (cudaMemsetAsync(ctr, 0, sizeof(Counters), s) != cudaSuccess) return MPS_E_CUDA;
    if (cudaMemcpyAsync(ditem, &d, sizeof(DevItem), cudaMemcpyHostToDevice, s) != cudaSuccess) return MPS_E_CUDA;
    if (launch_sieve(sa, tables, surv, nullptr, kNoAllocOdds, ctr, s) != cudaSuccess) return MPS_E_CUDA;
    if (launch_prep(pa, ctr, num_sms * 4, s) != cudaSuccess) return MPS_E_CUDA;
    if (launch_bsgs(ba, ctr, bgrid, s) != cudaSuccess) return MPS_E_CUDA;
    if (launch_order(oa, ctr, num_sms * 2, s) != cudaSuccess) return MPS_E_CUDA;
    Counters h;
    if (cudaMemcpyAsync(&h, ctr, sizeof(Counters), cudaMemcpyDeviceToHost, s) != cudaSuccess) return MPS_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MPS_E_CUDA;
    if (h.status & kStatusOrderFailed) return MPS_E_CUDA;
    if (h.status & (kStatusSurvivorOverflow | kStatusEntryOverflow | kStatusRelationOverflow)) {
        // denser than the scratch holds: split the range (no allocation)
        if (hi - lo < 64) return MPS_E_CAPACITY;
        const u64 mid = lo + (hi - lo) / 2;
        if (int r = run_pass(base, lo, mid, d, tbits, num_sms, sink)) return r;
        return run_pass(base, mid, hi, d, tbits, num_sms, sink);
    }
    const u64 nr = h.relations;
    if (nr && cudaMemcpy(g_host_rel, rel, nr * sizeof(RawRelation), cudaMemcpyDeviceToHost) != cudaSuccess)
        return MPS_E_CUDA;
    for (u64 i = 0; i < nr; ++i) {
        if (g_host_rel[i].q == ~0ull) continue;
        if (sink.n < sink.cap) {
            sink.out[sink.n].p = g_host_rel[i].p;
            sink.out[sink.n].M = g_host_rel[i].M;
            sink.out[sink.n].q = g_host_rel[i].q;
        }
        ++sink.n;
    }
    return MPS_OK;
}

}  // namespace

extern "C" int mps_chunk_relations_noalloc(uint64_t lo, uint64_t hi, const mps_item* item, mps_relation* out,
                                           size_t cap, size_t* n_out) {
    if (n_out) *n_out = 0;
    if (!out && cap) return MPS_E_ARG;
    if (lo >= hi) return MPS_OK;
    if (hi > (1ull << 62) || hi - lo > kNoAllocMaxSpan) return MPS_E_RANGE;
    DevItem d;
    u32 tbits = 0;
    if (int r = item_constants(item, &d, &tbits)) return r;
    int code = MPS_OK;
    unsigned char* base = scratch_for_current_device(&code);
    if (!base) return code;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return MPS_E_CUDA;
    Sink sink{out, cap, 0};
    if (int r = run_pass(base, lo, hi, d, tbits, sms, sink)) return r;
    if (n_out) *n_out = sink.n;
    if (sink.n > cap) return MPS_E_CAPACITY;
    std::sort(out, out + sink.n, [](const mps_relation& a, const mps_relation& b) { return a.p < b.p; });
    return MPS_OK;
}
