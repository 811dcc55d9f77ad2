// mps_item.cuh -- host-side construction of one item's device constants.
//
// Shared by the context entry points (mps_capi.cu) and the allocation-free
// entry point (mps_noalloc.cu).  Everything here is plain host integer code.
#pragma once

#include "../../include/mps_gpu.h"
#include "mps_common.cuh"

#include <cstring>

namespace mps {

inline u64 gcd_host(u64 a, u64 b) {
    while (b) {
        const u64 t = a % b;
        a = b;
        b = t;
    }
    return a;
}

constexpr u64 kMaxSplit = 1ull << 28;       // largest split modulus (at most 9 distinct primes)

// The split modulus Q of a tuning value: 0 -> lcm(cm, B) for the first B of
// kSplitBases whose lcm stays within 2^28 (5040 when none does); 1 ->
// lcm(cm, 2), the reference's plain-method filter (Gpu.hpp:247-298: the
// Legendre test and the gcd(mod, p-1)-th power test); anything else as given.
// Every prime l of Q with l | p - 1 splits a prime's exponents into l classes
// and keeps one, so a larger Q leaves fewer BSGS steps (about 1/(l-1) of the
// primes gain a factor l); the prep pays a longer walk for them.
constexpr u64 kSplitBases[] = {232792560ull, 720720ull, 5040ull};   // 2^4 3^2 5 7 11 13 17 19; to 13; to 7
inline u64 split_modulus(u32 class_modulus, u64 cm) {
    if (class_modulus == 0) {
        for (u64 base : kSplitBases) {
            const u64 l = cm / gcd_host(cm, base) * base;
            if (l <= kMaxSplit) return l;
        }
        return 5040;
    }
    if (class_modulus == 1) return cm % 2 == 0 ? cm : 2 * cm;
    return class_modulus;
}

// Validates an item the way load_worktodo does (Config.hpp:156-190), plus the
// GPU path's range P1 <= 2^62, and fills every DevItem field except the
// baby-step cap max_baby.  Returns MPS_OK, or an MPS_E_* code with *why set.
inline int item_constants(const mps_item* it, u32 class_modulus, u32 index, DevItem* d, const char** why) {
    *why = "";
    if (!it) return *why = "item is NULL", MPS_E_ARG;
    if (it->P0 >= it->P1) return *why = "requires P0 < P1", MPS_E_ARG;
    if (it->P1 > (1ull << 62)) return *why = "P1 must not exceed 2^62", MPS_E_RANGE;
    if (it->N0 >= it->N1) return *why = "requires N0 < N1", MPS_E_ARG;
    if ((unsigned __int128)((__int128)it->N1 - it->N0) > 10000000ull)
        return *why = "range N1-N0 exceeds 10 million", MPS_E_RANGE;
    const u64 cm = it->mod == 0 ? 1 : it->mod;
    if (it->res >= cm) return *why = "class must satisfy 0 <= res < mod", MPS_E_ARG;
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
    const u64 Q = split_modulus(class_modulus, cm);
    // Q <= 2^28 has at most 9 distinct prime factors (2*3*5*...*29 > 2^28)
    if (Q < 2 || Q > kMaxSplit || (Q & 1)) return *why = "class_modulus must be even and <= 2^28", MPS_E_ARG;
    d->Q = (u32)Q;
    d->Q_rcp = ~0ull / Q;
    u64 x = Q;
    for (u64 l = 2; l * l <= x; ++l) {
        if (x % l) continue;
        d->qf_l[d->qf_n++] = (u32)l;
        while (x % l == 0) x /= l;
    }
    if (x > 1) d->qf_l[d->qf_n++] = (u32)x;
    d->cmQ = (u32)(cm % Q);
    d->nsQ = (u32)(d->n_start % Q);
    d->item_index = index;
    d->baby_scale = kDefaultBabyScale;
    // the quadratic-character prefilter needs 0 < |b|, |c| < 2^32
    const unsigned __int128 lim = (unsigned __int128)1 << 32;
    if (babs > 0 && babs < lim && cabs > 0 && cabs < lim) {
        d->qr_on = 1;
        const u64 mag[2] = {(u64)babs, (u64)cabs};
        const u32 neg[2] = {b < 0 ? 1u : 0u, c > 0 ? 1u : 0u};     // x = b and x = -c
        for (int k = 0; k < 2; ++k) {
            const u32 tz = (u32)__builtin_ctzll(mag[k]);
            d->qr_neg[k] = neg[k];
            d->qr_k[k] = tz;
            d->qr_o[k] = (u32)(mag[k] >> tz);
            d->qr_rcp[k] = ~0ull / d->qr_o[k];
        }
    }
    return MPS_OK;
}

}  // namespace mps
