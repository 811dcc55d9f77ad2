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
// start of each pass.  Calls that overlap on one GPU (two host threads
// calling at once for the same device) race on that device's array and must
// not be made; calls on different devices use different arrays and may
// overlap.  The work is queued on the calling thread's per-thread default
// stream (cudaStreamPerThread), so it neither waits for nor blocks other
// streams of the device, and the host waits only for that stream.  No
// cudaMalloc, cudaFree, cudaMallocHost or other allocating routine is called,
// on the device or the host.
#include "../../include/mps_gpu.h"
#include "mps_item.cuh"
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

// Keys the fingerprint words of a 4 << tb byte table hold at the default fill.
u32 noalloc_holds(u32 tb) { return std::max<u32>(((1u << (tb - 1)) * kDefaultFill) >> 8, 1); }

// The item's device constants with the default tuning: the split modulus
// and the baby-step sizing of the regular entry points (fingerprint words at
// the default fill, 2^11 words at most).
int noalloc_item(const mps_item* it, DevItem* d, u32* tbits) {
    const char* why = "";
    if (int r = item_constants(it, 0, 0, d, &why)) return r;
    const u64 m_opt = (u64)std::ceil(std::sqrt((double)std::max<u64>(d->K, 1)));
    u32 tb = 6;
    while (noalloc_holds(tb) < m_opt && tb < 11) ++tb;
    *tbits = tb;
    d->max_baby = std::min<u32>(noalloc_holds(tb), kMaxBaby);
    return MPS_OK;
}

u32 prime_count_below_sqrt(u64 hi) {
    u32 n = 0;
    while (n < kSievePrimes && (u64)g_sp[n] * g_sp[n] < hi) ++n;
    return n;
}

// Raw relations are read back through a small buffer on the caller's stack.
constexpr u64 kReadBatch = 128;

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
    const cudaStream_t s = cudaStreamPerThread;

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
    pa.m_cap = std::min<u32>(noalloc_holds(tbits), kMaxBaby);
    pa.m_round = 64;                                         // one warp, two chains
    pa.prime_below = kSievedPrimeBelow;                      // survivors of the sieve
    BsgsArgs ba{};
    ba.ent = ent;
    ba.ent_cap = kNoAllocEntries;
    ba.rel = rel;
    ba.rel_cap = kNoAllocRelations;
    ba.tbits = tbits;
    ba.warps_per_block = 4;
    ba.persistent = 1;
    ba.chains = 2;
    ba.table_kind = 0;
    ba.load_shift = kDefaultLoadShift;
    ba.fill = kDefaultFill;
    ba.max_p = hi;
    OrderArgs oa{};
    oa.rel = rel;
    oa.rel_cap = kNoAllocRelations;
    oa.items = ditem;
    oa.tables = tables;

    const size_t smem = bsgs_smem_bytes(tbits, 4, 0);
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
    if (h.status & (kStatusOrderFailed | kStatusBadLaunch)) return MPS_E_CUDA;
    if (h.status & (kStatusSurvivorOverflow | kStatusEntryOverflow | kStatusRelationOverflow)) {
        // denser than the scratch holds: split the range (no allocation)
        if (hi - lo < 64) return MPS_E_CAPACITY;
        const u64 mid = lo + (hi - lo) / 2;
        if (int r = run_pass(base, lo, mid, d, tbits, num_sms, sink)) return r;
        return run_pass(base, mid, hi, d, tbits, num_sms, sink);
    }
    const u64 nr = h.relations;
    RawRelation buf[kReadBatch];
    for (u64 i0 = 0; i0 < nr; i0 += kReadBatch) {
        const u64 k = std::min<u64>(kReadBatch, nr - i0);
        if (cudaMemcpyAsync(buf, rel + i0, k * sizeof(RawRelation), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return MPS_E_CUDA;
        for (u64 i = 0; i < k; ++i) {
            if (buf[i].q == ~0ull) continue;      // a composite survivor
            if (sink.n < sink.cap) {
                sink.out[sink.n].p = buf[i].p;
                sink.out[sink.n].M = buf[i].M;
                sink.out[sink.n].q = buf[i].q;
            }
            ++sink.n;
        }
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
    if (int r = noalloc_item(item, &d, &tbits)) return r;
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
