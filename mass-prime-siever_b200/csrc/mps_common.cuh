// mps_common.cuh -- shared types of the sm_100a siever kernels.
//
// Device-side layout of one Factor= work item, the BSGS entry handed from
// the prep stage to the solve stage, and the relation record.  Everything is
// plain 64-bit integer data; nothing here touches torch.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mps {

typedef unsigned long long u64;
typedef long long i64;
typedef unsigned int u32;

// Odd primes 3..65521 (6,541 of them): the sieving primes of the segment
// sieve (same set as gpu_sieve_primes, Math.hpp:342-358).
constexpr u32 kSievePrimes = 6541;
constexpr u32 kSieveMaxPrime = 65521;

// Moduli below this run the FP64-pipe arithmetic (exact for p < 2^49); larger
// ones 64-bit Montgomery.
constexpr u64 kFp64Limit = 1ull << 49;

// Largest baby-step count of one prime (a table of 2^13 slots at load 1/2).
constexpr u32 kMaxBaby = 4096;
// Measured on the B200 (C2 and C3 slices): a baby step (hash, insert) costs
// about twice a giant step (hash, probe), so m = 0.625 sqrt(jcount) beats the
// square root, and words filled to 0.625 keys overflow rarely enough.
constexpr u32 kDefaultBabyScale = 160;   // m = ceil(sqrt(jcount)) x 160/256
constexpr u32 kDefaultFill = 160;        // fingerprint words: 0.625 keys per word on average

// Item constants, precomputed on the host once per item (all integer, exact).
struct DevItem {
    u64 babs_hi, babs_lo;  // |b| as 128-bit magnitude
    u64 cabs_hi, cabs_lo;  // |c|
    u32 b_neg, c_neg;      // signs
    i64 N0_raw;            // N0 as given (the p | b relation reports it, Math.hpp:496-502)
    i64 N1_raw;            // N1 as given (small-prime path, Math.hpp:506)
    u64 N0;                // max(N0, 0)  (Math.hpp:390)
    u64 N1;
    u64 cm;                // class modulus (>= 1)
    u64 n_start;           // smallest in-class n >= N0 (Math.hpp:393)
    u64 K;                 // in-class n in [n_start, N1): n = n_start + cm*k, k < K
    u32 has_work;          // K > 0
    u32 Q;                 // power-residue split modulus: g = gcd(Q, p - 1)
    u64 Q_rcp;             // floor((2^64 - 1) / Q)
    u32 cmQ;               // cm mod Q
    u32 nsQ;               // n_start mod Q
    u32 max_baby;          // cap on the baby-step count m of this item (<= kMaxBaby)
    u32 baby_scale;        // m = ceil(ceil(sqrt(jcount)) * baby_scale / 256) before the caps
    u32 item_index;
    u32 qf_n;              // prime factors of Q: qf_l[0..qf_n)
    u32 qf_l[9];
    // Quadratic-character prefilter (both |b| and |c| below 2^32): for x = b
    // and x = -c, x = (-1)^neg 2^k o with o odd; rcp = floor((2^64-1) / o).
    u32 qr_on;
    u32 qr_neg[2], qr_k[2], qr_o[2];
    u64 qr_rcp[2];
};

// One prime that reached the discrete-log stage: solve G0 * B^j == t (mod p)
// for the smallest j in [0, jcount).  Plain residues in [0, p).
struct Entry {
    u64 p;
    u64 t;                // -c
    u64 G0;               // b^n_first
    u64 B;                // b^L
    u64 Bm;               // B^m
    u64 n_first;          // smallest candidate n (n == r mod L, n >= N0)
    u64 L;                // n = n_first + j*L
    u64 jcount;
    u32 m;                // baby steps (<= kMaxBaby)
    u32 item;             // item index (batched runs)
};

// A relation before its order is known (q == 0 means "compute it").
struct RawRelation {
    u64 p, M, q;
    u32 item;
    u32 pad;
};

// Per-run device counters (one cache line each to keep atomics apart).
struct Counters {
    unsigned long long survivors;  u64 pad0[7];
    unsigned long long entries;    u64 pad1[7];
    unsigned long long relations;  u64 pad2[7];
    unsigned long long work_next;  u64 pad3[7];
    unsigned long long status;     u64 pad4[7];   // nonzero: an error bit set by a kernel
    unsigned long long primes;     u64 pad5[7];   // prime count (counting kernel only)
    unsigned long long steps;      u64 pad6[7];   // baby + giant steps executed by the BSGS
    unsigned long long prep_next;  u64 pad7[7];   // next survivor the prep's warps claim
    unsigned long long baby;       u64 pad8[7];   // the baby steps among `steps`
};

// Status bits a kernel may set (host turns them into error codes).
constexpr u64 kStatusSurvivorOverflow = 1ull << 0;
constexpr u64 kStatusEntryOverflow    = 1ull << 1;
constexpr u64 kStatusRelationOverflow = 1ull << 2;
constexpr u64 kStatusOrderFailed      = 1ull << 3;
constexpr u64 kStatusBadLaunch        = 1ull << 4;   // an entry the launch's kernel cannot take (host sizing error)

}  // namespace mps
