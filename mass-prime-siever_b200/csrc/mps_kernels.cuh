// mps_kernels.cuh -- launchers of the sm_100a siever kernels (mps_kernels.cu).
#pragma once

#include "mps_common.cuh"

namespace mps {

// Sieving-prime tables (device, built once per context).
struct SieveTables {
    const u32* sp;      // odd primes 3..65521
    const u64* rcp;     // floor((2^64 - 1) / q)
    const u64* inv;     // q^-1 mod 2^64
};

// Segment sieve of the odd numbers of [lo, hi) by the odd primes <= 65521:
// every survivor (an odd v >= 3 with no odd prime factor q <= min(65521,
// sqrt(hi)) other than itself) is appended to surv[].  include_two adds 2.
struct SieveArgs {
    u64 lo_odd;        // first odd >= max(lo, 3)
    u64 n_odds;        // odd numbers to sieve
    u64 hi;            // exclusive bound
    u32 include_two;
    u32 n_primes;      // sieving primes to use (those with q*q < hi, at most 6541)
    u32 item;          // item index stored with the survivors
};

// seg_words: segment bitmap words (1024, 2048 or 4096; 32 odd numbers each)
constexpr u32 kDefaultSegWords = 2048;
cudaError_t launch_sieve(const SieveArgs& a, const SieveTables& t, u64* surv, u32* surv_item, u64 surv_cap,
                         Counters* ctr, cudaStream_t s, u32 seg_words = kDefaultSegWords);

// A wave: several runs (odd ranges of possibly different items) sieved by
// one launch; kept in device memory so that a captured graph is replayable.
constexpr u32 kMaxRuns = 512;
struct SieveRun {
    u64 lo_odd;        // first odd >= max(lo, 3)
    u64 n_odds;
    u64 seg_begin;     // index of this run's first segment in the wave
    u64 hi;            // end of the run's integer range (lo .. hi)
    u32 n_primes;
    u32 include_two;
    u32 item;
    u32 pad;
};

// Device-resident state of one item: every P below p_done is sieved once the
// wave that covered it has committed; n_rel relations found, the first rel_cap
// of them kept in rel_buf (the item's reservation in a server's device pool;
// nullptr when the relations are not kept on the device).
struct ItemState {
    unsigned long long p_done;
    unsigned long long n_rel;
    unsigned long long waves;
    unsigned long long rel_cap;
    RawRelation* rel_buf;
    unsigned long long pad[3];
};
struct WaveDesc {
    u32 n_runs;
    u32 pad;
    u64 total_segs;
    SieveRun runs[kMaxRuns];
};
// After a wave: advance each run's item to the run's end, count relations.
cudaError_t launch_commit(const WaveDesc* w, const RawRelation* rel, const Counters* ctr, u64 rel_cap,
                          ItemState* st, cudaStream_t s);
// A run of an overflowed wave, redone on the host path: p_done = max(p_done, hi),
// its n relations rel[0..n) appended to the item's state.
cudaError_t launch_state_add(ItemState* st, u32 item, u64 hi, const RawRelation* rel, u64 n, cudaStream_t s);
// The wave's runs' seg_begin must count segments of seg_words * 32 odd numbers.
cudaError_t launch_sieve_wave(const WaveDesc* w, const SieveTables& t, u64* surv, u32* surv_item, u64 surv_cap,
                              Counters* ctr, int grid, cudaStream_t s, u32 seg_words = kDefaultSegWords);

// Prep: filters, primality screen and BSGS set-up for every survivor.
struct PrepArgs {
    const u64* surv;
    u64 surv_cap;
    const u32* surv_item;      // nullptr: every survivor belongs to `item0`
    u32 item0;
    const DevItem* items;
    Entry* ent;
    u64 ent_cap;
    RawRelation* rel;
    u64 rel_cap;
    u32 full_mr;               // 1: 12-base Miller-Rabin on every survivor that passes the filters
    u32 m_cap;                 // baby steps per prime at most (what the launch's BSGS tables hold)
    u32 m_round;               // baby steps rounded up to a multiple of this (the BSGS iteration width)
    u64 prime_below;           // survivors below this are prime (sieved by every prime up to their
                               // square root: 65521^2 for the sieve's survivors, 0 for caller-given numbers)
};
constexpr u64 kSievedPrimeBelow = (u64)kSieveMaxPrime * kSieveMaxPrime;
cudaError_t launch_prep(const PrepArgs& a, Counters* ctr, int grid, cudaStream_t s);

// Exact BSGS, one warp per entry.
struct BsgsArgs {
    const Entry* ent;
    u64 ent_cap;
    RawRelation* rel;
    u64 rel_cap;
    u32 tbits;                 // baby-step table of 2^tbits slots per warp
    u32 warps_per_block;
    u32 persistent;            // 1: work-stealing warps; 0: one warp per entry
    u32 chains;                // FP64 solve: independent chains per lane (1, 2, 4)
    u64 max_p;                 // largest p of the entries (>= 2^49: integer solve)
    u32 table_kind;            // FP64 solve: 0 = fingerprint words, 1 = 32-bit slots, 2 = 16-bit slots
    u32 load_shift;            // table kind 2: at most 2^-load_shift of a prime's slots are used
    u32 lanes;                 // table kind 2: lanes per prime, 32 (a warp) or 16 / 8 (groups; every
                               // entry must have p < 2^49, max_p > 0 and < 2^49 or the caller's guarantee)
    u32 fill;                  // table kinds 0 and 3: a prime's table has at least m * 256 / fill words
                               // (1..256; 0 counts as 256), within the launch's 2^(tbits-1)
};
constexpr u32 kDefaultLoadShift = 2;
cudaError_t launch_bsgs(const BsgsArgs& a, Counters* ctr, int grid, cudaStream_t s);
cudaError_t bsgs_reserve_smem(size_t smem);   // call before capturing a launch_bsgs

// Order q = ord_p(b) and the exact 12-base primality check of every relation.
struct OrderArgs {
    RawRelation* rel;
    u64 rel_cap;
    const DevItem* items;
    SieveTables tables;
};
cudaError_t launch_order(const OrderArgs& a, Counters* ctr, int grid, cudaStream_t s);

// Counts the primes among the survivors (exact 12-base test) into ctr->primes.
cudaError_t launch_count_primes(const u64* surv, u64 surv_cap, Counters* ctr, int grid, cudaStream_t s);

// Roofline probes: 256 x grid threads x 8 independent chains x iters operations.
cudaError_t launch_mmul_peak(u64 p, u32 iters, int grid, u64* sink, cudaStream_t s);
cudaError_t launch_imad_peak(u32 iters, int grid, u32* sink, cudaStream_t s);
cudaError_t launch_fmul_peak(u64 p, u32 iters, int grid, u64* sink, cudaStream_t s);
cudaError_t launch_smem_or_peak(u32 iters, int grid, u32* sink, cudaStream_t s);   // 256 x grid x 8 x iters

// Test hooks: raw kernels on given inputs.
cudaError_t launch_is_prime(const u64* n, u32* out, u64 count, cudaStream_t s);
cudaError_t launch_bsgs_direct(const u64* cases /* p,B,G0,t,jcount */, u64* j_out, u64 count, u32 tbits,
                               u32 table_kind, cudaStream_t s);
cudaError_t launch_order_direct(const u64* bp /* b,p pairs */, u64* q_out, u64 count, SieveTables t,
                                cudaStream_t s);

// Dynamic shared memory of a BSGS launch: 4 << tbits bytes of table per warp,
// and for table kind 3 one count byte per eight bytes of table.
size_t bsgs_smem_bytes(u32 tbits, u32 warps_per_block, u32 table_kind);

}  // namespace mps
