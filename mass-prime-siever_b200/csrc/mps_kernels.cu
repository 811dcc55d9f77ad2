// mps_kernels.cu -- the sm_100a kernels of the siever hot path.
//
//   k_sieve  segment sieve of the odd numbers by the odd primes <= 65521,
//            bitmap in shared memory, survivors compacted to global memory
//            (what psieve does, Gpu.hpp:385-455, sized for 148 SMs)
//   k_prep   per survivor: residues of b and -c, base-2 strong test,
//            power-residue split over g = gcd(Q, p - 1) (Gpu.hpp:465-589,
//            Math.hpp:410-433), BSGS set-up; staged through shared-memory
//            queues so that every stage runs with full warps
//   k_bsgs   exact baby-step giant-step, one warp per prime: baby-step table
//            of fingerprints + indices in shared memory, giant steps probed by
//            every lane, the smallest j found with a warp min-reduction
//            (the exact form of bsgs_wg / bsgs_wq, Gpu.hpp:329-383,600-650,
//            with run_bsgs's smallest-solution semantics, Math.hpp:439-483)
//   k_order  exact 12-base primality of each relation's p and q = ord_p(b)
//            (Math.hpp:209-251, 253-310), on the device
//
// All arithmetic is exact integer arithmetic; the relations equal those of
// the reference's CPU path.
#include "arith.cuh"
#include "mps_kernels.cuh"

#include <algorithm>
#include <mutex>

namespace mps {

constexpr u32 FULL = 0xFFFFFFFFu;

#ifndef MPS_BSGS_MINB
#define MPS_BSGS_MINB 3      // resident 256-thread BSGS blocks per SM the register budget is cut for
#endif

// ---------------------------------------------------------------- helpers --

// |x| mod p for the 128-bit magnitude hi:lo (shift-and-subtract for the rare
// wide values), then the sign.
__device__ __forceinline__ u64 residue128(u64 hi, u64 lo, u32 neg, u64 p) {
    u64 r;
    if (hi == 0) {
        r = lo < p ? lo : lo % p;
    } else {
        r = hi % p;
        for (int bit = 63; bit >= 0; --bit) {
            r = (r << 1) | ((lo >> bit) & 1ull);
            if (r >= p) r -= p;
        }
    }
    return (neg && r) ? p - r : r;
}

__device__ __forceinline__ u64 isqrt_ceil_dev(u64 x) {
    if (x == 0) return 0;
    u64 r = (u64)sqrt((double)x);
    while (r > 0 && r * r >= x) --r;
    while (r * r < x) ++r;
    return r;
}

__device__ __forceinline__ void emit_relation(u64 p, u64 M, u64 q, u32 item, RawRelation* rel, u64 cap,
                                              Counters* ctr) {
    const u64 slot = atomicAdd(&ctr->relations, 1ull);
    if (slot < cap) {
        RawRelation r;
        r.p = p; r.M = M; r.q = q; r.item = item; r.pad = 0;
        rel[slot] = r;
    } else {
        atomicOr(&ctr->status, kStatusRelationOverflow);
    }
}

// -------------------------------------------------------------- the sieve --

// A segment is W words of shared-memory bitmap (W * 32 odd numbers); W is a
// template parameter (1024, 2048 or 4096 words: 4, 8 or 16 KB), chosen per
// launch.  kSegWords is the default.
constexpr u32 kSegWords = 2048;
constexpr u32 kSieveThreads = 256;
constexpr u32 kNumPattern = 10;               // 3..31: whole-word patterns, no atomics
constexpr u32 kNumMedium = 171;               // primes below 1024: all threads share each prime

// Index j >= 0 of the first odd multiple v0 + 2j of q with v0 + 2j >= v0 (v0 odd).
__device__ __forceinline__ u32 first_odd_multiple(u64 v0, u32 q, u64 rcp) {
    const u64 qh = __umul64hi(v0, rcp);
    u64 r = v0 - qh * q;
    if (r >= q) r -= q;
    const u32 rr = (u32)r;
    return rr == 0 ? 0u : ((rr & 1u) ? (q - rr) >> 1 : q - (rr >> 1));
}

// Same, but never below q^2 (so q itself is never struck).
__device__ __forceinline__ u64 first_strike(u64 v0, u32 q, u64 rcp) {
    u64 j = first_odd_multiple(v0, q, rcp);
    const u64 qq = (u64)q * q;
    if (v0 + 2 * j < qq) j = (qq - v0) >> 1;
    return j;
}

template <u32 W>
struct SieveShared {
    u32 bits[W];
    u32 med_start[kNumMedium];
    u32 warp_sum[kSieveThreads / 32];
    unsigned long long block_base;
};

__device__ __forceinline__ void emit_two(u32 item, u64* surv, u32* surv_item, u64 cap, Counters* ctr) {
    const u64 slot = atomicAdd(&ctr->survivors, 1ull);
    if (slot < cap) {
        surv[slot] = 2;
        if (surv_item) surv_item[slot] = item;
    } else {
        atomicOr(&ctr->status, kStatusSurvivorOverflow);
    }
}

// One segment of len <= W * 32 odd numbers v0, v0 + 2, ... (v0 odd, >= 3),
// sieved by the first n_primes odd primes; survivors appended to surv[].
// Called by all threads of the block.
template <u32 W>
__device__ void sieve_segment(SieveShared<W>& sh, u64 v0, u32 len, u32 n_primes, u32 item, const SieveTables& t,
                              u64* surv, u32* surv_item, u64 cap, Counters* ctr) {
    constexpr u32 kSegOdds = W * 32, kWordsPerThread = W / kSieveThreads;
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const u32 n_med = min(n_primes, kNumMedium);
    // 1. primes 3..31: each thread writes whole words (pattern << offset).
    {
        u32 pat[kNumPattern], off[kNumPattern], step[kNumPattern], qs[kNumPattern];
#pragma unroll
        for (u32 k = 0; k < kNumPattern; ++k) {
            const u32 q = t.sp[k];
            qs[k] = q;
            u32 pm = 0;
            for (u32 b = 0; b < 32; b += q) pm |= 1u << b;
            pat[k] = pm;
            const u32 j0 = first_odd_multiple(v0, q, t.rcp[k]);
            int o = (int)j0 - (int)((32u * tid) % q);   // word w = tid first
            if (o < 0) o += (int)q;
            off[k] = (u32)o;
            step[k] = (32u * kSieveThreads) % q;
        }
        for (u32 w = tid; w < W; w += kSieveThreads) {
            u32 word = 0;
#pragma unroll
            for (u32 k = 0; k < kNumPattern; ++k) {
                word |= pat[k] << off[k];
                int o = (int)off[k] - (int)step[k];
                if (o < 0) o += (int)qs[k];
                off[k] = (u32)o;
            }
            sh.bits[w] = word;
        }
    }
    if (tid >= kNumPattern && tid < n_med)
        sh.med_start[tid] = (u32)min(first_strike(v0, t.sp[tid], t.rcp[tid]), (u64)kSegOdds);
    __syncthreads();
    // the pattern struck 3..31 themselves when they lie in this segment
    if (v0 <= 31 && tid < kNumPattern) {
        const u32 q = t.sp[tid];
        if (q >= v0) {
            const u32 i = (u32)((q - v0) >> 1);
            if (i < len) atomicAnd(&sh.bits[i >> 5], ~(1u << (i & 31)));
        }
    }
    // 2. primes 37..1021: all threads share each prime.
    for (u32 k = kNumPattern; k < n_med; ++k) {
        const u32 q = t.sp[k];
        for (u32 i = sh.med_start[k] + tid * q; i < len; i += kSieveThreads * q)
            atomicOr(&sh.bits[i >> 5], 1u << (i & 31));
    }
    // 3. primes 1031..65521: one thread per prime.
    for (u32 k = kNumMedium + tid; k < n_primes; k += kSieveThreads) {
        const u32 q = t.sp[k];
        const u64 j = first_strike(v0, q, t.rcp[k]);
        for (u64 i = j; i < len; i += q) atomicOr(&sh.bits[(u32)i >> 5], 1u << ((u32)i & 31));
    }
    __syncthreads();

    // 4. survivors: contiguous words per thread, block scan, one global atomic.
    const u32 w0 = tid * kWordsPerThread;
    u32 mine = 0;
#pragma unroll
    for (u32 k = 0; k < kWordsPerThread; ++k) {
        const u32 w = w0 + k;
        u32 x = ~sh.bits[w];
        const u32 first = w * 32;
        if (first >= len) x = 0;
        else if (len - first < 32) x &= (1u << (len - first)) - 1u;
        mine += __popc(x);
    }
    u32 incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(FULL, incl, o);
        if (lane >= (u32)o) incl += y;
    }
    if (lane == 31) sh.warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        u32 ws = lane < kSieveThreads / 32 ? sh.warp_sum[lane] : 0;
        u32 wincl = ws;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const u32 y = __shfl_up_sync(FULL, wincl, o);
            if (lane >= (u32)o) wincl += y;
        }
        if (lane < kSieveThreads / 32) sh.warp_sum[lane] = wincl - ws;   // exclusive
        if (lane == kSieveThreads / 32 - 1) sh.block_base = atomicAdd(&ctr->survivors, (unsigned long long)wincl);
    }
    __syncthreads();
    u64 pos = sh.block_base + sh.warp_sum[warp] + (incl - mine);
    for (u32 k = 0; k < kWordsPerThread; ++k) {
        const u32 w = w0 + k;
        u32 x = ~sh.bits[w];
        const u32 first = w * 32;
        if (first >= len) x = 0;
        else if (len - first < 32) x &= (1u << (len - first)) - 1u;
        while (x) {
            const u32 b = __ffs(x) - 1;
            x &= x - 1;
            if (pos < cap) {
                surv[pos] = v0 + 2ull * (first + b);
                if (surv_item) surv_item[pos] = item;
            }
            ++pos;
        }
    }
    if (pos > cap) atomicOr(&ctr->status, kStatusSurvivorOverflow);
    __syncthreads();
}

template <u32 W>
__global__ void __launch_bounds__(kSieveThreads) k_sieve(SieveArgs a, SieveTables t, u64* surv, u32* surv_item,
                                                         u64 cap, Counters* ctr) {
    constexpr u32 kSegOdds = W * 32;
    __shared__ SieveShared<W> sh;
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.include_two) emit_two(a.item, surv, surv_item, cap, ctr);
    for (u64 seg = blockIdx.x; seg * kSegOdds < a.n_odds; seg += gridDim.x) {
        const u64 base = seg * kSegOdds;
        sieve_segment(sh, a.lo_odd + 2 * base, (u32)min((u64)kSegOdds, a.n_odds - base), a.n_primes, a.item, t, surv,
                      surv_item, cap, ctr);
    }
}

// The same over a wave of runs (ranges of possibly different items), read
// from device memory so that a captured graph can be replayed per wave.
template <u32 W>
__global__ void __launch_bounds__(kSieveThreads) k_sieve_wave(const WaveDesc* w, SieveTables t, u64* surv,
                                                              u32* surv_item, u64 cap, Counters* ctr) {
    constexpr u32 kSegOdds = W * 32;
    __shared__ SieveShared<W> sh;
    const u32 n_runs = w->n_runs;
    const u64 total = w->total_segs;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (u32 r = 0; r < n_runs; ++r)
            if (w->runs[r].include_two) emit_two(w->runs[r].item, surv, surv_item, cap, ctr);
    for (u64 seg = blockIdx.x; seg < total; seg += gridDim.x) {
        u32 lo = 0, hi = n_runs;                        // last run with seg_begin <= seg
        while (hi - lo > 1) {
            const u32 mid = (lo + hi) >> 1;
            if (w->runs[mid].seg_begin <= seg) lo = mid;
            else hi = mid;
        }
        const SieveRun& run = w->runs[lo];
        const u64 base = (seg - run.seg_begin) * kSegOdds;
        if (base >= run.n_odds) continue;               // (a run with no odd numbers)
        sieve_segment(sh, run.lo_odd + 2 * base, (u32)min((u64)kSegOdds, run.n_odds - base), run.n_primes, run.item, t,
                      surv, surv_item, cap, ctr);
    }
}

// ------------------------------------------------------------ the fields --

// Two exact arithmetics behind one interface: FP64 (p < 2^49, the FP64 pipe)
// and 64-bit Montgomery (p < 2^62, the integer pipe).  V is the value type;
// key() gives the canonical integer (the table key) of a canonical value;
// eq(a, c) compares a product (or one()) with a canonical value c without
// leaving the field's representation.

struct FieldF {
    typedef double V;
    Fp64 f;
    __device__ __forceinline__ void init(u64 p) { f.init(p); }
    __device__ __forceinline__ V mul(V a, V b) const { return f.mul(a, b); }
    __device__ __forceinline__ V canon(V a) const { return f.canon(a); }          // units: (-p, p) -> [0, p)
    __device__ __forceinline__ u64 key(V c) const { return f.bits(c); }
    __device__ __forceinline__ u64 residue(V a) const { return f.residue(a); }   // any lazy value
    __device__ __forceinline__ V from_u64(u64 x) const { return (double)x; }
    __device__ __forceinline__ V one() const { return 1.0; }
    __device__ __forceinline__ V dbl(V a) const { return __dadd_rn(a, a); }      // (-p, p) -> (-2p, 2p)
    __device__ __forceinline__ V pow(V b, u64 e) const { return f.pow(b, e); }
    __device__ __forceinline__ bool eq(V a, V c) const { return a == c || a == c - f.p; }   // a in (-p, p)
};

struct FieldM {
    typedef u64 V;
    Mont M;
    u64 rr;
    __device__ __forceinline__ void init(u64 p) {
        M.init(p);
        rr = M.r2();
    }
    __device__ __forceinline__ V mul(V a, V b) const { return M.mul(a, b); }
    __device__ __forceinline__ V canon(V a) const { return M.norm(a); }
    __device__ __forceinline__ u64 key(V c) const { return c; }
    __device__ __forceinline__ u64 residue(V a) const { return M.from_mont(a); }
    __device__ __forceinline__ V from_u64(u64 x) const { return M.to_mont(x, rr); }
    __device__ __forceinline__ V one() const { return M.one; }
    __device__ __forceinline__ V dbl(V a) const { return M.dbl(a); }
    __device__ __forceinline__ V pow(V b, u64 e) const { return M.pow(b, e); }
    __device__ __forceinline__ bool eq(V a, V c) const { return a == c || a == c + M.p; }   // a in [0, 2p)
};

// --------------------------------------------------------------- the prep --

// p < 1000: the reference's direct BSGS over n in [0, m*m), m = ceil(sqrt(min(p, N1)))
// (Math.hpp:488-542), which yields the smallest such n; a walk gives the same n.
__device__ void small_prime(u64 p, u64 b_mod, u64 t, const DevItem& it, const PrepArgs& a, Counters* ctr) {
    const i64 lim = ((i64)p > it.N1_raw) ? it.N1_raw : (i64)p;
    if (lim <= 0) return;
    const u64 m = isqrt_ceil_dev((u64)lim);
    const u64 mm = m * m;
    u64 v = 1 % p;
    for (u64 n = 0; n < mm; ++n) {
        if (v == t) {
            emit_relation(p, n, 0, it.item_index, a.rel, a.rel_cap, ctr);
            return;
        }
        v = (v * b_mod) % p;
    }
}

// Strong probable-prime test to base 2 in field F (square-and-double).
template <class F>
__device__ __forceinline__ bool sprp2_f(const F& f, u64 p) {
    const u64 pm1 = p - 1;
    const int s = __ffsll((long long)pm1) - 1;
    const u64 d = pm1 >> s;
    int k = 63 - __clzll((long long)d);
    typename F::V x = f.dbl(f.one());               // 2 (top bit of d)
    for (--k; k >= 0; --k) {
        x = f.mul(x, x);
        if ((d >> k) & 1) x = f.dbl(x);
    }
    u64 y = f.residue(x);
    if (y == 1 || y == pm1) return true;
    for (int r = 1; r < s; ++r) {
        x = f.mul(x, x);
        y = f.residue(x);
        if (y == pm1) return true;
        if (y == 1) return false;
    }
    return false;
}

// Residues of b and -c for the survivor p, and the cases that never reach
// the field arithmetic: p | b (Math.hpp:383-385, 496-503), p < 1000
// (Math.hpp:488-542), p | c or no candidate n (Math.hpp:386-396).
// Returns true when p continues to the main path.
__device__ __forceinline__ bool prep_special(u64 p, const DevItem& it, const PrepArgs& a, Counters* ctr, u64& b_mod,
                                             u64& t) {
    b_mod = residue128(it.babs_hi, it.babs_lo, it.b_neg, p);
    const u64 c_mod = residue128(it.cabs_hi, it.cabs_lo, it.c_neg, p);
    t = c_mod == 0 ? 0 : p - c_mod;                     // -c mod p
    if (b_mod == 0) {
        if (t == 0) emit_relation(p, (u64)it.N0_raw, 1, it.item_index, a.rel, a.rel_cap, ctr);
        return false;
    }
    if (p < 1000) {
        small_prime(p, b_mod, t, it, a, ctr);
        return false;
    }
    return t != 0 && it.has_work;
}

// Quadratic-character prefilter (the reference's Jacobi filter, Gpu.hpp:
// 247-263, restated): b^n == t (mod p) forces (b/p)^n == (t/p).  With every
// in-class n == n_start (mod cm): for even cm the parity of n is fixed, so
// (b/p)^(n_start mod 2) must equal (t/p); for odd cm, (b/p) = 1 forces
// (t/p) = 1.  True when p can be dropped: a prime p then has no in-class
// solution, and a composite p never gives a relation.  Costs two Jacobi
// symbols of 32-bit numbers, before any modular exponentiation.
__device__ __forceinline__ bool qr_reject(u64 p, const DevItem& it) {
    if (!it.qr_on) return false;
    const int jb = jacobi_small(p, it.qr_neg[0], it.qr_k[0], it.qr_o[0], it.qr_rcp[0]);
    const int jt = jacobi_small(p, it.qr_neg[1], it.qr_k[1], it.qr_o[1], it.qr_rcp[1]);
    if (jb == 0 || jt == 0) return false;              // p shares a factor with b or c: the exact path decides
    if ((it.cm & 1) == 0) return (it.n_start & 1) ? jb != jt : jt != 1;
    return jb == 1 && jt != 1;
}

// e = (p - 1) / g exactly, g | p - 1.
__device__ __forceinline__ u64 exact_quotient(u64 pm1, u32 g) {
    const int tz = __ffs(g) - 1;
    return (pm1 >> tz) * (0 - Mont::neg_inverse((u64)(g >> tz)));
}

__device__ __forceinline__ u32 gcd_Q(const DevItem& it, u64 pm1) {
    const u64 qh = __umul64hi(pm1, it.Q_rcp);
    u32 rem = (u32)(pm1 - qh * it.Q);
    if (rem >= it.Q) rem -= it.Q;
    return gcd32(it.Q, rem);
}

// Stage 2: with g = gcd(Q, p - 1) and e = (p - 1) / g, w = b^e and u = t^e
// are g-th roots of unity and b^n == t forces w^n == u, i.e. n == r (mod d),
// d = ord(w) -- or there is no solution.  Returns 0 (no solution), 1 (d, r
// found by a walk of at most `walk` steps) or 2 (longer: deferred, with the
// residues of w and u in w_out, u_out for stage 2b).
template <class F>
__device__ __forceinline__ int power_split(const F& f, u64 p, u64 b_mod, u64 t, const DevItem& it, u32 walk, u32& d,
                                           u32& r, u64& w_out, u64& u_out) {
    typedef typename F::V V;
    const u64 pm1 = p - 1;
    const u32 g = gcd_Q(it, pm1);
    const u64 e = exact_quotient(pm1, g);
    V u = f.one(), w = f.one(), bu = f.from_u64(t), bw = f.from_u64(b_mod);
    for (u64 x = e; x; x >>= 1) {                      // two exponentiations, interleaved
        if (x & 1) {
            u = f.mul(u, bu);
            w = f.mul(w, bw);
        }
        bu = f.mul(bu, bu);
        bw = f.mul(bw, bw);
    }
    const V uc = f.canon(u), one = f.one();
    V x = one;
    bool found = false;
    const u32 lim = min(g, walk);
    for (u32 k = 0; k < lim; ++k) {                    // discrete log in <w>
        if (!found && f.eq(x, uc)) {
            r = k;
            found = true;
        }
        x = f.mul(x, w);
        if (f.eq(x, one)) {
            d = k + 1;
            return found ? 1 : 0;
        }
    }
    if (lim == g) return 0;
    w_out = f.residue(w);
    u_out = f.residue(u);
    return 2;
}

// Stage 2b: the same split for long orders, one prime power of g at a time,
// from stage 2's w and u (residues): w_l = w^(g/l^c), u_l = u^(g/l^c) in the
// l^c-th roots of unity, a walk of at most l^c steps each, combined by the
// Chinese remainder theorem.
template <class F>
__device__ bool power_split_pp(const F& f, u64 p, u64 w_res, u64 u_res, const DevItem& it, u32& d, u32& r) {
    typedef typename F::V V;
    const u32 g = gcd_Q(it, p - 1);
    const V w = f.from_u64(w_res), u = f.from_u64(u_res);
    d = 1;
    r = 0;
    for (u32 i = 0; i < it.qf_n; ++i) {
        const u32 l = it.qf_l[i];
        if (g % l) continue;
        u32 lc = l;
        while (g % (lc * l) == 0) lc *= l;
        const u32 k = g / lc;
        const V wl = f.pow(w, k), uc = f.canon(f.pow(u, k)), one = f.one();
        V x = one;
        bool found = false;
        u32 xr = 0, dl = lc;
        for (u32 y = 0; y < lc; ++y) {
            if (!found && f.eq(x, uc)) {
                xr = y;
                found = true;
            }
            x = f.mul(x, wl);
            if (f.eq(x, one)) {
                dl = y + 1;
                break;
            }
        }
        if (!found) return false;
        // r' == r (mod d), r' == xr (mod dl); d, dl coprime
        u32 step = 0;                                      // d * dl <= g <= Q <= 2^28
        while ((r + d * step) % dl != xr) ++step;
        r += d * step;
        d *= dl;
    }
    return true;
}

// Stage 3: n = n_start + cm*k (in class) with n == r (mod d); the BSGS set-up
// for G0 * B^j == t, G0 = b^n_first, B = b^L, j < jcount.
template <class F>
__device__ void bsgs_setup(const F& f, u64 p, u64 b_mod, u64 t, const DevItem& it, u32 d, u32 r, const PrepArgs& a,
                           Counters* ctr) {
    typedef typename F::V V;
    // the smallest k0 >= 0 with n_start + cm*k0 == r (mod d): k0*cmd == want
    // (mod d) is solvable iff h = gcd(cmd, d) divides want, and then its
    // solutions are k0 + per*i with per = d/h, k0 = (want/h)(cmd/h)^-1 mod per
    const u32 cmd = it.cmQ % d;                        // d | Q
    const u32 want = (r + d - it.nsQ % d) % d;
    const u32 h = gcd32(cmd, d);                       // gcd(0, d) = d
    if (want % h) return;
    const u32 per = d / h;                             // period of k
    const u32 k0 = (u32)((u64)(want / h) * inv_mod32((cmd / h) % per, per) % per);
    if (k0 >= it.K) return;
    u64 jcount = ((u32)it.K - k0 + per - 1) / per;     // K < 2^32 (N1 - N0 <= 10^7)
    if (jcount > p) jcount = p;                        // ord(B) < p (Math.hpp:398-400)
    const u64 L = it.cm * per;
    const u64 n_first = it.n_start + it.cm * k0;
    // G0 = b^n_first and B = b^L from one chain of squarings of b
    V sq = f.from_u64(b_mod), gv = f.one(), Bv = f.one();
    for (u64 e1 = n_first, e2 = L; e1 | e2;) {
        if (e1 & 1) gv = f.mul(gv, sq);
        if (e2 & 1) Bv = f.mul(Bv, sq);
        e1 >>= 1;
        e2 >>= 1;
        if (e1 | e2) sq = f.mul(sq, sq);
    }
    const u64 G0 = f.residue(gv);
    if (G0 == t) {                                     // j = 0
        emit_relation(p, n_first, 0, it.item_index, a.rel, a.rel_cap, ctr);
        return;
    }
    if (jcount <= 1) return;
    u32 m = (u32)isqrt_ceil_dev(jcount);
    if (it.baby_scale != 256) m = max(1u, (u32)(((u64)m * it.baby_scale + 255) >> 8));
    // a whole number of baby iterations (lanes x chains per prime): the last
    // iteration's lanes then all insert, and the extra baby steps save giant steps
    if (a.m_round > 1) m = (m + a.m_round - 1) / a.m_round * a.m_round;
    if (m > it.max_baby) m = it.max_baby;
    if (m > a.m_cap) m = a.m_cap;                      // never more than the launch's tables hold
    const u64 Bm = f.residue(f.pow(Bv, m));
    const u64 slot = atomicAdd(&ctr->entries, 1ull);
    if (slot >= a.ent_cap) {
        atomicOr(&ctr->status, kStatusEntryOverflow);
        return;
    }
    Entry e;
    e.p = p; e.t = t; e.G0 = G0; e.B = f.residue(Bv); e.Bm = Bm;
    e.n_first = n_first; e.L = L; e.jcount = jcount; e.m = m; e.item = it.item_index;
    a.ent[slot] = e;
}

template <class F>
__device__ __forceinline__ bool stage1(u64 p, const PrepArgs& a) {
    if (p < a.prime_below) return true;                // the sieve removed every composite below this
    F f;
    f.init(p);
    if (!sprp2_f(f, p)) return false;
    return !a.full_mr || is_prime64(p);
}

constexpr u32 kPrepThreads = 256;
constexpr u32 kWalk = 48;                              // stage-2 walk before deferring

// Warp-aggregated push onto a shared-memory queue.
__device__ __forceinline__ u32 queue_slot(u32* count, bool want) {
    const u32 bal = __ballot_sync(FULL, want);
    if (!bal) return 0;
    const u32 lane = threadIdx.x & 31;
    const int leader = __ffs(bal) - 1;
    u32 base = 0;
    if ((int)lane == leader) base = atomicAdd(count, __popc(bal));
    base = __shfl_sync(FULL, base, leader);
    return base + __popc(bal & ((1u << lane) - 1));
}

// The prep: one persistent kernel without block barriers.  Every warp claims
// 32 survivors at a time and carries them through the stages on its own,
// with three warp-private queues in shared memory between the stages
// (survivors that passed stage 1; primes with their (d, r) for stage 3;
// primes deferred to stage 2b).  A queue is drained whenever it holds 32
// entries, so every stage runs with full warps, and a warp never waits for
// another; the partial queues are drained at the end.  A queue never holds
// more than 63 entries: a stage pushes at most 32 into a queue that held
// fewer than 32.
constexpr u32 kPrepWarps = kPrepThreads / 32;

struct PrepQueues {
    u64 p1[64];
    u32 i1[64];
    u64 p2[64];
    u32 i2[64], d2[64], r2[64];
    u64 pd[64];
    u64 wd[64], ud[64];                            // stage 2's w and u of a deferred prime
    u32 id[64];
};

// Appends the lanes with want to a warp queue of n entries (n warp-uniform).
__device__ __forceinline__ void qpush(bool want, u32& n, u32* slot_out) {
    const u32 lane = threadIdx.x & 31;
    const u32 bal = __ballot_sync(FULL, want);
    *slot_out = n + __popc(bal & ((1u << lane) - 1));
    n += __popc(bal);
}

template <class F>
__device__ __forceinline__ int split_in(const DevItem& it, u64 p, u32& d, u32& r, u64& w, u64& u) {
    F f;
    f.init(p);
    const u64 bm = residue128(it.babs_hi, it.babs_lo, it.b_neg, p);
    const u64 t = p - residue128(it.cabs_hi, it.cabs_lo, it.c_neg, p);
    return power_split(f, p, bm, t, it, kWalk, d, r, w, u);
}

template <class F>
__device__ __forceinline__ bool split_pp_in(const DevItem& it, u64 p, u64 w, u64 u, u32& d, u32& r) {
    F f;
    f.init(p);
    return power_split_pp(f, p, w, u, it, d, r);
}

template <class F>
__device__ __forceinline__ void setup_in(const DevItem& it, u64 p, u32 d, u32 r, const PrepArgs& a, Counters* ctr) {
    F f;
    f.init(p);
    const u64 bm = residue128(it.babs_hi, it.babs_lo, it.b_neg, p);
    const u64 t = p - residue128(it.cabs_hi, it.cabs_lo, it.c_neg, p);
    bsgs_setup(f, p, bm, t, it, d, r, a, ctr);
}

__global__ void __launch_bounds__(kPrepThreads) k_prep(PrepArgs a, Counters* ctr) {
    __shared__ PrepQueues qs[kPrepWarps];
    PrepQueues& Q = qs[threadIdx.x >> 5];
    const u32 lane = threadIdx.x & 31;
    const u64 n_surv = min((u64)*(volatile unsigned long long*)&ctr->survivors, a.surv_cap);
    u32 n1 = 0, n2 = 0, nd = 0;                          // queue lengths (warp-uniform)
    bool inputs = true;
    for (;;) {
        if (n2 >= 32 || (!inputs && n1 == 0 && nd == 0 && n2 > 0)) {
            // stage 3: class combination and the BSGS set-up
            const u32 cnt = min(n2, 32u);
            if (lane < cnt) {
                const u32 k = n2 - cnt + lane;
                const u64 p = Q.p2[k];
                const DevItem& it = a.items[Q.i2[k]];
                if (p < kFp64Limit) setup_in<FieldF>(it, p, Q.d2[k], Q.r2[k], a, ctr);
                else setup_in<FieldM>(it, p, Q.d2[k], Q.r2[k], a, ctr);
            }
            n2 -= cnt;
            __syncwarp();
            continue;
        }
        if (nd >= 32 || (!inputs && n1 == 0 && nd > 0)) {
            // stage 2b: long orders, one prime power at a time
            const u32 cnt = min(nd, 32u);
            bool ok = false;
            u32 d = 1, r = 0, item = 0;
            u64 p = 0;
            if (lane < cnt) {
                const u32 k = nd - cnt + lane;
                p = Q.pd[k];
                item = Q.id[k];
                const DevItem& it = a.items[item];
                const u64 w = Q.wd[k], u = Q.ud[k];
                ok = p < kFp64Limit ? split_pp_in<FieldF>(it, p, w, u, d, r) : split_pp_in<FieldM>(it, p, w, u, d, r);
            }
            nd -= cnt;
            __syncwarp();
            u32 s2;
            qpush(ok, n2, &s2);
            if (ok) {
                Q.p2[s2] = p;
                Q.i2[s2] = item;
                Q.d2[s2] = d;
                Q.r2[s2] = r;
            }
            __syncwarp();
            continue;
        }
        if (n1 >= 32 || (!inputs && n1 > 0)) {
            // stage 2: power-residue split with a short walk
            const u32 cnt = min(n1, 32u);
            int res = 0;
            u32 d = 1, r = 0, item = 0;
            u64 p = 0, w = 0, u = 0;
            if (lane < cnt) {
                const u32 k = n1 - cnt + lane;
                p = Q.p1[k];
                item = Q.i1[k];
                const DevItem& it = a.items[item];
                res = p < kFp64Limit ? split_in<FieldF>(it, p, d, r, w, u) : split_in<FieldM>(it, p, d, r, w, u);
            }
            n1 -= cnt;
            __syncwarp();
            u32 s2, sd;
            qpush(res == 1, n2, &s2);
            qpush(res == 2, nd, &sd);
            if (res == 1) {
                Q.p2[s2] = p;
                Q.i2[s2] = item;
                Q.d2[s2] = d;
                Q.r2[s2] = r;
            } else if (res == 2) {
                Q.pd[sd] = p;
                Q.wd[sd] = w;
                Q.ud[sd] = u;
                Q.id[sd] = item;
            }
            __syncwarp();
            continue;
        }
        if (!inputs) break;
        // stage 1: claim 32 survivors; special cases, the quadratic-character
        // prefilter, then the base-2 strong test
        u64 first = 0;
        if (lane == 0) first = atomicAdd(&ctr->prep_next, 32ull);
        first = __shfl_sync(FULL, first, 0);
        if (first >= n_surv) {
            inputs = false;
            continue;
        }
        const u64 k = first + lane;
        bool keep = false;
        u64 p = 0;
        u32 item = a.item0;
        if (k < n_surv) {
            p = a.surv[k];
            if (a.surv_item) item = a.surv_item[k];
            u64 bm, t;
            if (prep_special(p, a.items[item], a, ctr, bm, t) && !qr_reject(p, a.items[item]))
                keep = p < kFp64Limit ? stage1<FieldF>(p, a) : stage1<FieldM>(p, a);
        }
        u32 s1;
        qpush(keep, n1, &s1);
        if (keep) {
            Q.p1[s1] = p;
            Q.i1[s1] = item;
        }
        __syncwarp();
    }
}

// --------------------------------------------------------------- the BSGS --
//
// One warp per prime.  The baby-step table holds a 16-bit fingerprint per
// slot (0 = empty; linear probing); a giant value whose fingerprint matches
// is resolved exactly by recomputing the baby steps, which is rare (true
// solutions, and fingerprint collisions at ~2^-15 per compare).

__device__ __forceinline__ void table_hash(u64 key, u32 tbits, u32& slot, u32& fp) {
    const u32 lo = (u32)key, hi = (u32)(key >> 32);
    const u32 x = (lo ^ (hi * 0x9E3779B1u)) * 0x85EBCA6Bu;
    slot = x >> (32 - tbits);
    fp = (x & 0xFFFFu) | 1u;
}

__device__ __forceinline__ void table_insert(unsigned short* tab, u32 mask, u32 tbits, u64 key) {
    u32 s, fp;
    table_hash(key, tbits, s, fp);
    while (atomicCAS(&tab[s], (unsigned short)0, (unsigned short)fp) != 0) s = (s + 1) & mask;
}

__device__ __forceinline__ bool table_maybe(const unsigned short* tab, u32 mask, u32 tbits, u64 key) {
    u32 s, fp;
    table_hash(key, tbits, s, fp);
    for (;;) {
        const u32 e = tab[s];
        if (e == fp) return true;
        if (e == 0) return false;
        s = (s + 1) & mask;
    }
}

// Smallest i in [lo, limit) with key(t * B^i) == key, or -1 (warp-cooperative;
// tbl = t * B^lane, B32 = B^32).
template <class F>
__device__ __noinline__ int find_baby_index(const F& f, typename F::V tbl, typename F::V B32, u32 lo, u32 limit, u64 key) {
    const u32 lane = threadIdx.x & 31;
    typename F::V v = tbl;
    for (u32 base = 0; base < limit; base += 32) {
        const u32 i = base + lane;
        const bool hit = i >= lo && i < limit && f.key(f.canon(v)) == key;
        const u32 bal = __ballot_sync(FULL, hit);
        if (bal) return (int)(base + __ffs(bal) - 1);
        v = f.mul(v, B32);
    }
    return -1;
}

// A solve's step counts for its caller: giant steps in the high 32 bits,
// baby steps in the low 32 (baby <= kMaxBaby, giant <= jcount <= 10^7).
__device__ __forceinline__ u64 pack_steps(u64 baby, u64 giant) { return (giant << 32) | baby; }

// Solves one entry with the 32 lanes of the calling warp; returns the
// smallest j (< jcount) or ~0ull.  Two interleaved chains per lane: baby
// indices i = l + 64k and l + 32 + 64k, giant steps g = 1 + l + 64k and
// 33 + l + 64k.
template <class F>
__device__ u64 solve_entry(const Entry& e, unsigned short* tab, u32 tbits, u64* steps_out) {
    typedef typename F::V V;
    const u32 lane = threadIdx.x & 31;
    F f;
    f.init(e.p);
    const u32 m = e.m;
    const u32 T = 1u << tbits, mask = T - 1;
    const V B = f.from_u64(e.B), Bm = f.from_u64(e.Bm), tv = f.from_u64(e.t), G0 = f.from_u64(e.G0);
    const u64 tkey = f.key(f.canon(tv));

    // lane powers by an inclusive scan: xb = B^(l+1), xg = Bm^(l+1)
    V xb = B, xg = Bm;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const V yb = __shfl_up_sync(FULL, xb, off), yg = __shfl_up_sync(FULL, xg, off);
        if (lane >= (u32)off) {
            xb = f.mul(xb, yb);
            xg = f.mul(xg, yg);
        }
    }
    const V B32 = __shfl_sync(FULL, xb, 31), Bm32 = __shfl_sync(FULL, xg, 31);
    V bl = __shfl_up_sync(FULL, xb, 1);
    if (lane == 0) bl = f.one();                       // B^l
    const V B64 = f.mul(B32, B32), Bm64 = f.mul(Bm32, Bm32);
    const V tbl = f.mul(tv, bl);                       // t B^l
    V baby0 = tbl, baby1 = f.mul(tbl, B32);
    V gi0 = f.mul(G0, xg), gi1 = f.mul(gi0, Bm32);

    uint4* t4 = reinterpret_cast<uint4*>(tab);
    for (u32 k = lane; k < T / 8; k += 32) t4[k] = make_uint4(0, 0, 0, 0);
    __syncwarp();

    // baby steps t*B^i, stopping at a cycle B^d == 1 (d < m)
    u32 cyc = 0;
    u64 steps = 0, baby_steps = 0;
    for (u32 base = 0; base < m; base += 64) {
        const u32 i0 = base + lane, i1 = base + 32 + lane;
        const u64 k0 = f.key(f.canon(baby0)), k1 = f.key(f.canon(baby1));
        const u32 b0 = __ballot_sync(FULL, i0 > 0 && i0 < m && k0 == tkey);
        const u32 b1 = __ballot_sync(FULL, i1 < m && k1 == tkey);
        u32 lim = m;
        if (b0 | b1) {
            cyc = b0 ? base + __ffs(b0) - 1 : base + 32 + __ffs(b1) - 1;
            lim = cyc;
        }
        if (i0 < lim) table_insert(tab, mask, tbits, k0);
        if (i1 < lim) table_insert(tab, mask, tbits, k1);
        steps += min(64u, lim - base);
        baby_steps += min(64u, lim - base);
        if (cyc) break;
        baby0 = f.mul(baby0, B64);
        baby1 = f.mul(baby1, B64);
    }
    __syncwarp();

    u64 best = ~0ull;
    if (cyc) {
        // ord(B) = cyc < m: the answer is the j in [1, cyc) with G0 == t*B^(cyc-j)
        // (j = 0 was ruled out by the prep); t*B^i, i < cyc, are distinct.
        const int i = find_baby_index(f, tbl, B32, 1, cyc, f.key(f.canon(G0)));
        if (i > 0) best = cyc - (u32)i;
    } else {
        const u64 G = (e.jcount - 1 + m - 1) / m;      // giant steps g = 1..G cover j in [1, G*m]
        for (u64 base = 0; base < G; base += 64) {
            const u64 g0 = base + 1 + lane, g1 = base + 33 + lane;
            const u64 k0 = f.key(f.canon(gi0)), k1 = f.key(f.canon(gi1));
            const bool h0 = g0 <= G && table_maybe(tab, mask, tbits, k0);
            const bool h1 = g1 <= G && table_maybe(tab, mask, tbits, k1);
            const u32 bal0 = __ballot_sync(FULL, h0), bal1 = __ballot_sync(FULL, h1);
            steps += min((u64)64, G - base);
            if (bal0 | bal1) {
                // candidates in increasing g: the first exact one is the smallest j
                u64 jb = ~0ull;
                for (int pass = 0; pass < 2 && jb == ~0ull; ++pass) {
                    u32 bal = pass == 0 ? bal0 : bal1;
                    while (bal && jb == ~0ull) {
                        const int src = __ffs(bal) - 1;
                        bal &= bal - 1;
                        const u64 kk = __shfl_sync(FULL, pass == 0 ? k0 : k1, src);
                        const u64 gg = base + (pass == 0 ? 1 : 33) + (u64)src;
                        const int i = find_baby_index(f, tbl, B32, 0, m, kk);
                        if (i >= 0) jb = gg * m - (u64)i;
                    }
                }
                if (jb != ~0ull) {
                    best = jb;
                    break;
                }
            }
            gi0 = f.mul(gi0, Bm64);
            gi1 = f.mul(gi1, Bm64);
        }
    }
    __syncwarp();
    if (steps_out) *steps_out = pack_steps(baby_steps, steps - baby_steps);
    return best < e.jcount ? best : ~0ull;
}

// ---- the FP64 solve (p < 2^49): the hot loop of the whole path ----
//
// Table: 2^tbits 32-bit slots per warp.  A key's home slot is the top tbits
// of a multiplicative hash h of the canonical value's two 32-bit halves; the
// slot word is (h & ~1) | 2 (never 0) plus bit 0, the overflow bit, set on a
// home slot when a key homed there had to move further (linear probing).  A
// probe therefore reads one slot: a match, an empty slot, or an occupied slot
// without the overflow bit all end it; only an overflowed home (rare at the
// load factors used) walks the chain, in a ballot-guarded slow path.  A match
// is resolved exactly by recomputation (ffind_baby): true solutions, and hash
// collisions at about 2^-20 per compare.

__device__ __forceinline__ u32 fhash(double v) {
    return (u32)(__double2loint(v) ^ __double2hiint(v)) * 0x9E3779B1u;
}

__device__ __forceinline__ u32 fword(u32 h) { return (h & ~3u) | 2u; }

__device__ __forceinline__ void ftable_insert(u32* tab, u32 mask, u32 shift, u32 h) {
    u32 s = h >> shift;
    const u32 w = fword(h);
    if (atomicCAS(&tab[s], 0u, w) == 0u) return;
    atomicOr(&tab[s], 1u);                         // a key homed here moves on
    do s = (s + 1) & mask;
    while (atomicCAS(&tab[s], 0u, w) != 0u);
}

// Continues a probe past an overflowed home slot s.
__device__ __forceinline__ bool ftable_walk(const u32* tab, u32 mask, u32 s, u32 w) {
    for (;;) {
        s = (s + 1) & mask;
        const u32 e = tab[s];
        if (e == 0u) return false;
        if ((e & ~1u) == w) return true;
    }
}

// Smallest i in [lo, limit) with t * B^i == v (canonical doubles compared
// exactly); -1 when there is none.  Warp-cooperative: tbl = t * B^lane.
__device__ __noinline__ int ffind_baby(const Fp64& f, double tbl, double B32, u32 lo, u32 limit, double v) {
    const u32 lane = threadIdx.x & 31;
    double x = tbl;
    for (u32 base = 0; base < limit; base += 32) {
        const u32 i = base + lane;
        const bool hit = i >= lo && i < limit && f.canon(x) == v;
        const u32 bal = __ballot_sync(FULL, hit);
        if (bal) return (int)(base + __ffs(bal) - 1);
        x = f.mul(x, B32);
    }
    return -1;
}

// CH interleaved chains per lane: baby index i = lane + 32c + 32*CH*k,
// giant step g = 1 + lane + 32c + 32*CH*k.
template <int CH>
__device__ u64 solve_fp64(const Entry& e, u32* tab, u32 tbits, u64* steps_out) {
    const u32 lane = threadIdx.x & 31;
    Fp64 f;
    f.init(e.p);
    const u32 m = e.m;
    const u32 jc = (u32)e.jcount;                      // jcount <= 10^7
    // this prime's table: 2^tb slots for m baby steps (load <= ~1/5), at most the launch's
    tbits = min(tbits, max(6u, 32u - __clz(5 * m - 1)));
    const u32 mask = (1u << tbits) - 1, shift = 32 - tbits;
    const double B = (double)e.B, Bm = (double)e.Bm, tv = (double)e.t, G0 = (double)e.G0;

    double xb = B, xg = Bm;                            // B^(l+1), Bm^(l+1)
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double yb = __shfl_up_sync(FULL, xb, off), yg = __shfl_up_sync(FULL, xg, off);
        if (lane >= (u32)off) {
            xb = f.mul(xb, yb);
            xg = f.mul(xg, yg);
        }
    }
    const double B32 = __shfl_sync(FULL, xb, 31), Bm32 = __shfl_sync(FULL, xg, 31);
    double bl = __shfl_up_sync(FULL, xb, 1);
    if (lane == 0) bl = 1.0;
    double Bstep = B32, Gstep = Bm32;                  // B^(32 CH), Bm^(32 CH)
#pragma unroll
    for (int c = 1; c < CH; c <<= 1) {
        Bstep = f.mul(Bstep, Bstep);
        Gstep = f.mul(Gstep, Gstep);
    }
    const double tbl = f.mul(tv, bl);
    double bx[CH], gx[CH];
    bx[0] = tbl;
    gx[0] = f.mul(G0, xg);
#pragma unroll
    for (int c = 1; c < CH; ++c) {
        bx[c] = f.mul(bx[c - 1], B32);
        gx[c] = f.mul(gx[c - 1], Bm32);
    }

    uint4* t4 = reinterpret_cast<uint4*>(tab);
    for (u32 k = lane; k <= mask / 4; k += 32) t4[k] = make_uint4(0, 0, 0, 0);
    __syncwarp();

    // baby steps, stopping at a cycle B^d == 1 (d < m)
    u32 cyc = 0, baby_done = m;
    for (u32 base = 0; base < m; base += 32 * CH) {
        double cv[CH];
        u32 cb = 0;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            cv[c] = f.canon(bx[c]);
            const u32 i = base + 32 * c + lane;
            const u32 bc = __ballot_sync(FULL, i > 0 && i < m && cv[c] == tv);
            if (bc && !cb) cb = base + 32 * c + __ffs(bc) - 1;
        }
        const u32 lim = cb ? cb : m;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const u32 i = base + 32 * c + lane;
            if (i < lim) ftable_insert(tab, mask, shift, fhash(cv[c]));
        }
        if (cb) {
            cyc = cb;
            baby_done = cb;
            break;
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) bx[c] = f.mul(bx[c], Bstep);
    }
    __syncwarp();

    u64 best = ~0ull;
    u32 giant_done = 0;
    if (cyc) {
        const int i = ffind_baby(f, tbl, B32, 1, cyc, G0);
        if (i > 0) best = cyc - (u32)i;
    } else {
        const u32 G = (jc - 1 + m - 1) / m;            // g = 1..G covers j in [1, G*m]
        giant_done = G;
        for (u32 base = 0; base < G; base += 32 * CH) {
            double cv[CH];
            u32 hit = 0;
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                cv[c] = f.canon(gx[c]);
                const u32 h = fhash(cv[c]);
                const u32 s0 = h >> shift;
                const u32 w1 = (h & ~3u) | 3u;         // the slot word with the overflow bit forced
                const u32 e = tab[s0];
                bool m1 = (e | 1u) == w1;
                if (!m1 && (e & 1u)) m1 = ftable_walk(tab, mask, s0, w1 & ~1u);
                hit |= m1 ? (1u << c) : 0u;
            }
            if (__any_sync(FULL, hit)) {
                u32 bal[CH];
#pragma unroll
                for (int c = 0; c < CH; ++c)
                    bal[c] = __ballot_sync(FULL, ((hit >> c) & 1u) && base + 32 * c + lane + 1 <= G);
                // candidates in increasing g: the first exact one gives the smallest j
                u64 jb = ~0ull;
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    u32 bb = bal[c];
                    while (bb && jb == ~0ull) {
                        const int src = __ffs(bb) - 1;
                        bb &= bb - 1;
                        const double v = __shfl_sync(FULL, cv[c], src);
                        const u64 g = base + 32 * c + (u32)src + 1;
                        const int i = ffind_baby(f, tbl, B32, 0, m, v);
                        if (i >= 0) jb = g * m - (u64)i;
                    }
                }
                if (jb != ~0ull) {
                    best = jb;
                    giant_done = min(G, base + 32 * CH);
                    break;
                }
            }
#pragma unroll
            for (int c = 0; c < CH; ++c) gx[c] = f.mul(gx[c], Gstep);
        }
    }
    __syncwarp();
    if (steps_out) *steps_out = pack_steps(baby_done, giant_done);
    return best < e.jcount ? best : ~0ull;
}

// ---- the FP64 solve with a fingerprint table (the default) ----
//
// Table: 2^tw 64-bit words per warp, each holding up to four 16-bit halves
// filled in order (half k = bits 16k..16k+15): bit 15 of a half marks it
// used, bits 0..13 hold a 14-bit fingerprint of the key; bit 14 of half 0 is
// the word's overflow bit, set when a key homed at this word found it full
// and moved on (linear probing over words).  The home word is the top tw bits
// of the key's multiplicative hash h, the fingerprint the next 14 bits.  For
// m baby steps tw = ceil(log2(m * 256 / fill)), so a word holds at most
// fill/256 keys on average (fill 160: 0.6, and about 0.1% of the words
// overflow).  A probe reads one word and tests the four halves at once
// (fq_probe); a home with its overflow bit set also counts as a candidate.
// The next giant value is multiplied before the probe of the current one, so
// the multiply's latency overlaps the shared-memory load.  Candidates leave the
// hot loop: the lane walks the overflow chain, and a fingerprint found is
// resolved exactly by recomputation (ffind_baby).  Compared with one 32-bit
// key per slot this stores 2.5x as many baby steps in the same shared memory
// and never walks inside the hot loop.

constexpr u64 kQValid = 0x8000800080008000ull;

// log2 of the words a prime with m baby steps gets: at least m * 256 / fill
// words (fill 1..256; 0 counts as 256) and at least 32, at most 2^(tbits-1).
__device__ __forceinline__ u32 fq_words_log(u32 m, u32 fill, u32 tbits, u32 extra_shift) {
    const u32 f = fill - 1u < 256u ? fill : 256u;
    const u32 keys = max(m, 2u) * 256u;                // m <= 4096: fits 32 bits
    u32 t = 32u - __clz(max(m, 2u) - 1);               // 2^t >= m; 2^t f >= 256 m needs at most 8 more
    while ((f << t) < keys) ++t;                       // no division: f << t <= 2^28
    return min(tbits - 1, max(5u, t + extra_shift));
}
constexpr u32 kQOvf = 0x4000u;

__device__ __forceinline__ u32 fq_pattern(u32 h, u32 tw) {
    return ((h >> (18 - tw)) & 0x3FFFu) | 0x8000u;
}

__device__ __forceinline__ bool fq_word_has(u64 w, u32 pat) {
    const u32 lo = (u32)w & ~kQOvf, hi = (u32)(w >> 32);
    return (lo & 0xFFFFu) == pat || (lo >> 16) == pat || (hi & 0xFFFFu) == pat || (hi >> 16) == pat;
}

__device__ __forceinline__ void fq_insert(unsigned long long* tab, u32 mask, u32 home, u32 pat) {
    volatile unsigned long long* vt = tab;
    u32 s = home;
    unsigned long long w = vt[s];
    for (;;) {
        if (w >> 63) {                               // full: move on (marking the home once)
            if (s == home && !(w & kQOvf)) atomicOr(&tab[home], (unsigned long long)kQOvf);
            s = (s + 1) & mask;
            w = vt[s];
            continue;
        }
        const u32 k = __popcll(w & kQValid);
        const unsigned long long nw = w | ((unsigned long long)pat << (16 * k));
        const unsigned long long old = atomicCAS(&tab[s], w, nw);
        if (old == w) return;
        w = old;
    }
}

// Whether the key (home, pat) is in the table: its home word, then the
// overflow chain up to the first word that is not full.
__device__ __forceinline__ bool fq_contains(const unsigned long long* tab, u32 mask, u32 home, u32 pat) {
    u64 w = tab[home];
    if (fq_word_has(w, pat)) return true;
    if (!(w & kQOvf)) return false;
    for (u32 s = (home + 1) & mask, n = 0; n <= mask; s = (s + 1) & mask, ++n) {
        w = tab[s];
        if (fq_word_has(w, pat)) return true;
        if (!(w >> 63)) return false;
    }
    return false;
}

// Table kind 3: the fingerprint words of kind 0 with a count byte per word
// (after the launch's words: one byte per eight of table).  Every chain's key
// with want claims the next half of its home word by one shared-memory atomic
// add on the word's count and writes its fingerprint with a plain 16-bit
// store (every claimed half is distinct).  A claim that finds the word full
// (count >= 4) is taken back at once, so a count rests at 4 at most and never
// passes 4 + 32 * CH in flight (a byte cannot wrap).  The rare keys whose home
// was full then walk on, word by word, in rounds of the whole warp, as in
// kind 0's walk; the overflow bits of their homes are set after every store
// of the call, so a store to half 0 never clears one.
__device__ __forceinline__ u32 fq_claim(unsigned char* cnt, u32 s) {
    const u32 sh = 8u * (s & 3u);
    u32* c32 = reinterpret_cast<u32*>(cnt) + (s >> 2);
    const u32 k = (atomicAdd(c32, 1u << sh) >> sh) & 0xFFu;
    if (k >= 4u) atomicSub(c32, 1u << sh);          // full: take the claim back
    return k;
}

template <int CH>
__device__ __forceinline__ void fq_insert_count(unsigned long long* tab, unsigned char* cnt, u32 mask, u32 want,
                                                const u32 (&home)[CH], const u32 (&pat)[CH]) {
    unsigned short* t16 = reinterpret_cast<unsigned short*>(tab);
    u32 k[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) k[c] = (want >> c) & 1u ? fq_claim(cnt, home[c]) : 0u;
    u32 pend = 0;                                      // bit c: chain c found its home full
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        if (!((want >> c) & 1u)) continue;
        if (k[c] < 4u) t16[4 * home[c] + k[c]] = (unsigned short)pat[c];
        else pend |= 1u << c;
    }
    if (!__any_sync(FULL, pend)) return;
    const u32 ovf = pend;
    u32 s[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) s[c] = (home[c] + 1) & mask;
    while (__any_sync(FULL, pend)) {
#pragma unroll
        for (int c = 0; c < CH; ++c) k[c] = (pend >> c) & 1u ? fq_claim(cnt, s[c]) : 4u;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            if (!((pend >> c) & 1u)) continue;
            if (k[c] < 4u) {
                t16[4 * s[c] + k[c]] = (unsigned short)pat[c];
                pend &= ~(1u << c);
            } else {
                s[c] = (s[c] + 1) & mask;
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int c = 0; c < CH; ++c)
        if ((ovf >> c) & 1u) atomicOr(reinterpret_cast<u32*>(tab) + 2 * home[c], kQOvf);
}

// The probe of a giant value: nonzero when a used half of the home word
// equals the fingerprint, or the word overflowed.  With x = word ^ pattern
// (both halves of the pattern), a 16-bit half of x is zero exactly when that
// half matches, and (x - 0x00010001) & ~x & 0x80008000 is then nonzero.  The
// caller ORs the probes of its chains and votes once per iteration.
__device__ __forceinline__ u32 fq_probe(const uint2* t2, u32 h, u32 shift, u32 tw) {
    const uint2 w = t2[h >> shift];
    const u32 rep = fq_pattern(h, tw) * 0x10001u;
    const u32 x0 = (w.x & ~kQOvf) ^ rep, x1 = w.y ^ rep;
    return (((x0 - 0x10001u) & ~x0) & 0x80008000u) | (((x1 - 0x10001u) & ~x1) & 0x80008000u) | (w.x & kQOvf);
}

// WI: baby steps inserted by fq_insert_count (table kind 3, count bytes
// after the words) instead of one compare-and-swap each (table kind 0); the
// words and the probes are the same.
template <int CH, bool WI>
__device__ u64 solve_fp64q(const Entry& e, unsigned long long* tab, u32 tbits, u32 fill, u64* steps_out) {
    const u32 lane = threadIdx.x & 31;
    Fp64 f;
    f.init(e.p);
    const u32 m = e.m;
    const u32 jc = (u32)e.jcount;                      // jcount <= 10^7
    // 2^tw words for m keys (at most fill/256 per word), within the launch's 2^(tbits-1) words
    const u32 tw = fq_words_log(m, fill, tbits, 0);
    const u32 mask = (1u << tw) - 1, shift = 32 - tw;
    const double B = (double)e.B, Bm = (double)e.Bm, tv = (double)e.t, G0 = (double)e.G0;

    double xb = B, xg = Bm;                            // B^(l+1), Bm^(l+1)
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double yb = __shfl_up_sync(FULL, xb, off), yg = __shfl_up_sync(FULL, xg, off);
        if (lane >= (u32)off) {
            xb = f.mul(xb, yb);
            xg = f.mul(xg, yg);
        }
    }
    const double B32 = __shfl_sync(FULL, xb, 31), Bm32 = __shfl_sync(FULL, xg, 31);
    double bl = __shfl_up_sync(FULL, xb, 1);
    if (lane == 0) bl = 1.0;
    double Bstep = B32, Gstep = Bm32;                  // B^(32 CH), Bm^(32 CH)
#pragma unroll
    for (int c = 1; c < CH; c <<= 1) {
        Bstep = f.mul(Bstep, Bstep);
        Gstep = f.mul(Gstep, Gstep);
    }
    const double tbl = f.mul(tv, bl);
    double bx[CH], gx[CH];
    bx[0] = tbl;
    gx[0] = f.mul(G0, xg);
#pragma unroll
    for (int c = 1; c < CH; ++c) {
        bx[c] = f.mul(bx[c - 1], B32);
        gx[c] = f.mul(gx[c - 1], Bm32);
    }

    unsigned char* cnt = reinterpret_cast<unsigned char*>(tab) + (4u << tbits);   // kind 3 only
    uint4* t4 = reinterpret_cast<uint4*>(tab);
#pragma unroll 4
    for (u32 k = lane; k <= mask / 2; k += 32) t4[k] = make_uint4(0, 0, 0, 0);
    if (WI)
        for (u32 k = lane; k <= mask / 16; k += 32) reinterpret_cast<uint4*>(cnt)[k] = make_uint4(0, 0, 0, 0);
    __syncwarp();

    // baby steps, stopping at a cycle B^d == 1 (d < m): t B^i == t for an
    // i in [1, m) is looked for with one vote per iteration, and located
    // exactly only when one is found
    u32 cyc = 0, baby_done = m;
    for (u32 base = 0; base < m; base += 32 * CH) {
        double cv[CH], nb[CH];
        bool hit = false;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            cv[c] = f.canon(bx[c]);
            nb[c] = f.mul(bx[c], Bstep);                   // the next value, independent of the insert
            hit |= base + 32 * c + lane - 1u < m - 1u && cv[c] == tv;
        }
        u32 cb = 0;
        if (__any_sync(FULL, hit)) {
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const u32 bc = __ballot_sync(FULL, base + 32 * c + lane - 1u < m - 1u && cv[c] == tv);
                if (bc && !cb) cb = base + 32 * c + __ffs(bc) - 1;
            }
        }
        const u32 lim = cb ? cb : m;
        if (WI) {
            u32 home[CH], pat[CH], want = 0;
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const u32 h = fhash(cv[c]);
                home[c] = h >> shift;
                pat[c] = fq_pattern(h, tw);
                if (base + 32 * c + lane < lim) want |= 1u << c;
            }
            fq_insert_count<CH>(tab, cnt, mask, want, home, pat);
        } else {
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const u32 h = fhash(cv[c]);
                if (base + 32 * c + lane < lim) fq_insert(tab, mask, h >> shift, fq_pattern(h, tw));
            }
        }
        if (cb) {
            cyc = cb;
            baby_done = cb;
            break;
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) bx[c] = nb[c];
    }
    __syncwarp();

    u64 best = ~0ull;
    u32 giant_done = 0;
    if (cyc) {
        const int i = ffind_baby(f, tbl, B32, 1, cyc, G0);
        if (i > 0) best = cyc - (u32)i;
    } else {
        const u32 G = (jc - 1 + m - 1) / m;            // g = 1..G covers j in [1, G*m]
        giant_done = G;
        const uint2* t2 = reinterpret_cast<const uint2*>(tab);
        for (u32 base = 0; base < G; base += 32 * CH) {
            double cv[CH], nx[CH];
            u32 hs[CH];
            u32 z = 0;
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                cv[c] = f.canon(gx[c]);
                hs[c] = fhash(cv[c]);
                nx[c] = f.mul(gx[c], Gstep);              // the next value, independent of the probe
                z |= fq_probe(t2, hs[c], shift, tw);
            }
            if (__any_sync(FULL, z)) {
                // the rare path: walk overflowed homes, then resolve exact matches in increasing g
                u32 real = 0;
#pragma unroll
                for (int c = 0; c < CH; ++c)
                    if (base + 32 * c + lane + 1 <= G && fq_probe(t2, hs[c], shift, tw) &&
                        fq_contains(tab, mask, hs[c] >> shift, fq_pattern(hs[c], tw)))
                        real |= 1u << c;
                u64 jb = ~0ull;
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    u32 bb = __ballot_sync(FULL, (real >> c) & 1u);
                    while (bb && jb == ~0ull) {
                        const int src = __ffs(bb) - 1;
                        bb &= bb - 1;
                        const double v = __shfl_sync(FULL, cv[c], src);
                        const u64 g = base + 32 * c + (u32)src + 1;
                        const int i = ffind_baby(f, tbl, B32, 0, m, v);
                        if (i >= 0) jb = g * m - (u64)i;
                    }
                }
                if (jb != ~0ull) {
                    best = jb;
                    giant_done = min(G, base + 32 * CH);
                    break;
                }
            }
#pragma unroll
            for (int c = 0; c < CH; ++c) gx[c] = nx[c];
        }
    }
    __syncwarp();
    if (steps_out) *steps_out = pack_steps(baby_done, giant_done);
    return best < e.jcount ? best : ~0ull;
}

// ---- the FP64 solve with a 16-bit slot table ----
//
// Table: 2^(tbits+1) 16-bit slots per warp (4 << tbits bytes), of which a
// prime with m baby steps uses 2^tw, tw = ceil(log2 m) + load_shift (load at
// most 2^-load_shift).  A key -- the canonical residue x of a baby step -- is
// hashed from the low 32 bits of x, which the FP64 pipe exposes with one add
// (x + 2^52 has x in its low mantissa bits): h = lo32(x) * kHashMul, a
// bijection of lo32(x).  The home slot is the top tw bits of h and holds the
// 15-bit fingerprint (h & 0x7FFF) | 1 (never 0; 0 is an empty slot).  Bit 15
// of a slot is its overflow flag, set when a key homed there found it taken
// and moved on (linear probing).  A probe reads its home slot only: equal
// fingerprints make a candidate; a set overflow flag sends the lane to the
// warp's slow path, which walks the chain.  Candidates are resolved exactly by
// recomputing the baby steps, so fingerprint collisions (about 2^-14 per
// occupied probe) never change a result.

constexpr u32 kHashMul = 0x9E3779B1u;

__device__ __forceinline__ u32 hkey_canon(double x) {          // x canonical in [0, p), p < 2^49
    return (u32)__double2loint(__dadd_rn(x, 4503599627370496.0)) * kHashMul;
}

__device__ __forceinline__ u32 hfp(u32 h) { return (h & 0x7FFFu) | 1u; }

__device__ __forceinline__ void h_insert(unsigned short* tab, u32 mask, u32 shift, u32 h) {
    u32 s = h >> shift;
    const unsigned short f = (unsigned short)hfp(h);
    if (atomicCAS(&tab[s], (unsigned short)0, f) == 0) return;
    atomicOr(reinterpret_cast<u32*>(tab) + (s >> 1), 0x8000u << (16 * (s & 1)));   // flag the home slot
    do s = (s + 1) & mask;
    while (atomicCAS(&tab[s], (unsigned short)0, f) != 0);
}

// Whether a key with hash h may be in the table: its home slot, then (when the
// home's overflow flag is set) the chain up to the first empty slot.
__device__ __forceinline__ bool h_contains(const unsigned short* tab, u32 mask, u32 shift, u32 h) {
    u32 s = h >> shift;
    const u32 f = hfp(h);
    u32 e = tab[s];
    if (((e ^ f) & 0x7FFFu) == 0) return true;
    if (!(e & 0x8000u)) return false;
    for (u32 n = 0; n < mask; ++n) {
        s = (s + 1) & mask;
        e = tab[s];
        if (e == 0) return false;
        if (((e ^ f) & 0x7FFFu) == 0) return true;
    }
    return false;
}

template <int CH>
__device__ u64 solve_fp64h(const Entry& e, unsigned short* tab, u32 tbits, u32 load_shift, u64* steps_out) {
    const u32 lane = threadIdx.x & 31;
    Fp64 f;
    f.init(e.p);
    const u32 m = e.m;
    const u32 jc = (u32)e.jcount;                      // jcount <= 10^7
    const u32 tw = min(tbits + 1, max(6u, 32u - __clz(max(m, 2u) - 1) + load_shift));
    const u32 mask = (1u << tw) - 1, shift = 32 - tw;
    const double B = (double)e.B, Bm = (double)e.Bm, tv = (double)e.t, G0 = (double)e.G0;

    double xb = B, xg = Bm;                            // B^(l+1), Bm^(l+1)
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double yb = __shfl_up_sync(FULL, xb, off), yg = __shfl_up_sync(FULL, xg, off);
        if (lane >= (u32)off) {
            xb = f.mul(xb, yb);
            xg = f.mul(xg, yg);
        }
    }
    const double B32 = __shfl_sync(FULL, xb, 31), Bm32 = __shfl_sync(FULL, xg, 31);
    double bl = __shfl_up_sync(FULL, xb, 1);
    if (lane == 0) bl = 1.0;
    double Bstep = B32, Gstep = Bm32;                  // B^(32 CH), Bm^(32 CH)
#pragma unroll
    for (int c = 1; c < CH; c <<= 1) {
        Bstep = f.mul(Bstep, Bstep);
        Gstep = f.mul(Gstep, Gstep);
    }
    const double tbl = f.mul(tv, bl);
    double bx[CH], gx[CH];
    bx[0] = tbl;
    gx[0] = f.mul(G0, xg);
#pragma unroll
    for (int c = 1; c < CH; ++c) {
        bx[c] = f.mul(bx[c - 1], B32);
        gx[c] = f.mul(gx[c - 1], Bm32);
    }

    uint4* t4 = reinterpret_cast<uint4*>(tab);
    for (u32 k = lane; k <= (mask >> 3); k += 32) t4[k] = make_uint4(0, 0, 0, 0);
    __syncwarp();

    // baby steps, stopping at a cycle B^d == 1 (d < m)
    u32 cyc = 0, baby_done = m;
    for (u32 base = 0; base < m; base += 32 * CH) {
        double cv[CH];
        u32 cb = 0;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            cv[c] = f.canon(bx[c]);
            const u32 i = base + 32 * c + lane;
            const u32 bc = __ballot_sync(FULL, i > 0 && i < m && cv[c] == tv);
            if (bc && !cb) cb = base + 32 * c + __ffs(bc) - 1;
        }
        const u32 lim = cb ? cb : m;
#pragma unroll
        for (int c = 0; c < CH; ++c)
            if (base + 32 * c + lane < lim) h_insert(tab, mask, shift, hkey_canon(cv[c]));
        if (cb) {
            cyc = cb;
            baby_done = cb;
            break;
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) bx[c] = f.mul(bx[c], Bstep);
    }
    __syncwarp();

    u64 best = ~0ull;
    u32 giant_done = 0;
    if (cyc) {
        const int i = ffind_baby(f, tbl, B32, 1, cyc, G0);
        if (i > 0) best = cyc - (u32)i;
    } else {
        const u32 G = (jc - 1 + m - 1) / m;            // g = 1..G covers j in [1, G*m]
        giant_done = G;
        for (u32 base = 0; base < G; base += 32 * CH) {
            u32 hs[CH];
            bool flag = false;
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                hs[c] = hkey_canon(f.canon(gx[c]));
                const u32 slot = tab[hs[c] >> shift];
                flag |= (((slot ^ hfp(hs[c])) & 0x7FFFu) == 0) | ((slot & 0x8000u) != 0);
            }
            if (__any_sync(FULL, flag)) {
                // the slow path: walk overflowed homes, then resolve candidates in increasing g
                u32 real = 0;
#pragma unroll
                for (int c = 0; c < CH; ++c)
                    if (base + 32 * c + lane + 1 <= G && h_contains(tab, mask, shift, hs[c])) real |= 1u << c;
                u64 jb = ~0ull;
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    u32 bb = __ballot_sync(FULL, (real >> c) & 1u);
                    while (bb && jb == ~0ull) {
                        const int src = __ffs(bb) - 1;
                        bb &= bb - 1;
                        const double v = __shfl_sync(FULL, f.canon(gx[c]), src);
                        const u64 g = base + 32 * c + (u32)src + 1;
                        const int i = ffind_baby(f, tbl, B32, 0, m, v);
                        if (i >= 0) jb = g * m - (u64)i;
                    }
                }
                if (jb != ~0ull) {
                    best = jb;
                    giant_done = min(G, base + 32 * CH);
                    break;
                }
            }
#pragma unroll
            for (int c = 0; c < CH; ++c) gx[c] = f.mul(gx[c], Gstep);
        }
    }
    __syncwarp();
    if (steps_out) *steps_out = pack_steps(baby_done, giant_done);
    return best < e.jcount ? best : ~0ull;
}

template <int CH, int QT>
__device__ __forceinline__ u64 solve_any(const Entry& e, void* tab, u32 tbits, u32 load_shift, u32 fill, u64* steps) {
    if (CH == 0 || e.p >= kFp64Limit) return solve_entry<FieldM>(e, (unsigned short*)tab, tbits + 1, steps);
    if (QT == 0) return solve_fp64q<CH ? CH : 1, false>(e, (unsigned long long*)tab, tbits, fill, steps);
    if (QT == 2) return solve_fp64h<CH ? CH : 1>(e, (unsigned short*)tab, tbits, load_shift, steps);
    if (QT == 3) return solve_fp64q<CH ? CH : 1, true>(e, (unsigned long long*)tab, tbits, fill, steps);
    return solve_fp64<CH ? CH : 1>(e, (u32*)tab, tbits, steps);
}

// Whether a prime's baby steps fit the table its solve will use (at most half
// of its keys' room), so that every insertion finds a free slot.
template <int CH, int QT>
__device__ __forceinline__ bool fits_table(const Entry& e, u32 tbits) {
    if (CH == 0 || e.p >= kFp64Limit) return e.m <= (1u << tbits);          // 2^(tbits+1) 16-bit slots
    if (QT == 0 || QT == 3) return e.m <= (1u << tbits);                    // 2^(tbits-1) words of four
    if (QT == 2) return e.m <= (1u << tbits);                               // 2^(tbits+1) 16-bit slots
    return e.m < (1u << tbits);                                            // 2^tbits 32-bit slots
}

// CH > 0: every entry has p < 2^49 (FP64 solve with CH chains per lane);
// CH == 0: any p (integer Montgomery solve).
template <int CH, int QT>
__global__ void __launch_bounds__(256, MPS_BSGS_MINB) k_bsgs(BsgsArgs a, Counters* ctr) {
    extern __shared__ __align__(16) u32 smem32[];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // per warp 4 << tbits bytes of table (kind 3: and one count byte per eight)
    u32* tab = smem32 + (size_t)warp * ((1u << a.tbits) + (QT == 3 ? (1u << a.tbits) / 8 : 0u));
    const u64 n_ent = min((u64)*(volatile unsigned long long*)&ctr->entries, a.ent_cap);
    u64 my_steps = 0, my_baby = 0;
    if (a.persistent) {
        // A warp claims the entry after the one it solves, and lanes 0..8 load
        // that entry's nine words while the current one is solved, so neither
        // the claim nor the load is waited for between entries.
        static_assert(sizeof(Entry) == 72, "entry staging assumes nine 64-bit words");
        u64 cur = 0;
        if (lane == 0) cur = atomicAdd(&ctr->work_next, 1ull);
        cur = __shfl_sync(FULL, cur, 0);
        u64 claim = 0;                                          // lane 0: the entry after cur
        if (lane == 0 && cur < n_ent) claim = atomicAdd(&ctr->work_next, 1ull);
        u64 stage = cur < n_ent && lane < 9 ? reinterpret_cast<const u64*>(a.ent + cur)[lane] : 0;
        while (cur < n_ent) {
            // the solve's fields; n_first, L and item are read again for a relation
            Entry e;
            e.p = __shfl_sync(FULL, stage, 0);
            e.t = __shfl_sync(FULL, stage, 1);
            e.G0 = __shfl_sync(FULL, stage, 2);
            e.B = __shfl_sync(FULL, stage, 3);
            e.Bm = __shfl_sync(FULL, stage, 4);
            e.n_first = 0;
            e.L = 0;
            e.jcount = __shfl_sync(FULL, stage, 7);
            e.m = (u32)__shfl_sync(FULL, stage, 8);             // little-endian: m, then item
            e.item = 0;
            const u64 idx = cur;
            const u64 next = __shfl_sync(FULL, claim, 0);
            stage = next < n_ent && lane < 9 ? reinterpret_cast<const u64*>(a.ent + next)[lane] : 0;
            if (lane == 0 && next < n_ent) claim = atomicAdd(&ctr->work_next, 1ull);
            cur = next;
            if (!fits_table<CH, QT>(e, a.tbits)) {              // host sizing error: never overfill a table
                if (lane == 0) atomicOr(&ctr->status, kStatusBadLaunch);
                continue;
            }
            u64 steps = 0;
            const u64 j = solve_any<CH, QT>(e, tab, a.tbits, a.load_shift, a.fill, &steps);
            if (lane == 0) {
                if (j != ~0ull) {
                    const Entry& g = a.ent[idx];
                    emit_relation(e.p, g.n_first + j * g.L, 0, g.item, a.rel, a.rel_cap, ctr);
                }
                my_steps += (steps & 0xFFFFFFFFull) + (steps >> 32);
                my_baby += steps & 0xFFFFFFFFull;
            }
        }
        if (lane == 0 && my_steps) {
            atomicAdd(&ctr->steps, (unsigned long long)my_steps);
            atomicAdd(&ctr->baby, (unsigned long long)my_baby);
        }
    } else {
        const u64 idx = (u64)blockIdx.x * a.warps_per_block + warp;
        if (idx >= n_ent) return;
        const Entry e = a.ent[idx];
        if (!fits_table<CH, QT>(e, a.tbits)) {
            if (lane == 0) atomicOr(&ctr->status, kStatusBadLaunch);
            return;
        }
        u64 steps = 0;
        const u64 j = solve_any<CH, QT>(e, tab, a.tbits, a.load_shift, a.fill, &steps);
        if (lane == 0) {
            if (j != ~0ull) emit_relation(e.p, e.n_first + j * e.L, 0, e.item, a.rel, a.rel_cap, ctr);
            atomicAdd(&ctr->steps, (unsigned long long)((steps & 0xFFFFFFFFull) + (steps >> 32)));
            atomicAdd(&ctr->baby, (unsigned long long)(steps & 0xFFFFFFFFull));
        }
    }
}

// ---- lanes per prime: L-lane groups, 32/L primes per warp in lockstep ----
//
// For primes with few baby and giant steps a whole warp per prime spends
// most of its time on per-prime set-up (the lane-power scan, the table
// clear).  Here a warp takes 32/L entries at once and each group of L lanes
// solves one with its own 16-bit slot table (a 1/(32/L) share of the warp's
// table memory); the loops run to the largest bound among the warp's primes
// with per-group predicates, so the groups never diverge.  Same tables, same
// exact resolution and the same smallest-j result as solve_fp64h.

// Smallest i in [lo, limit) with t * B^i == v within the group (-1: none).
// Warp-uniform control flow: a group with want == false only keeps pace.
template <int L>
__device__ int gfind_baby(const Fp64& f, double tbl, double BL, u32 lo, u32 limit, double v, bool want, u32 gl,
                          u32 gshift, u32 gbits) {
    const u32 lim_max = __reduce_max_sync(FULL, want ? limit : 0u);
    double x = tbl;
    int res = -1;
    for (u32 base = 0; base < lim_max; base += L) {
        const u32 i = base + gl;
        const bool hit = want && res < 0 && i >= lo && i < limit && f.canon(x) == v;
        const u32 gb = (__ballot_sync(FULL, hit) >> gshift) & gbits;
        if (gb && res < 0) res = (int)(base + __ffs(gb) - 1);
        if (__all_sync(FULL, !want || res >= 0 || base + L >= limit)) break;
        x = f.mul(x, BL);
    }
    return res;
}

template <int L, int CH>
__global__ void __launch_bounds__(256, MPS_BSGS_MINB) k_bsgs_groups(BsgsArgs a, Counters* ctr) {
    constexpr u32 NG = 32 / L;
    constexpr u32 NG_LOG = NG == 4 ? 2 : NG == 2 ? 1 : 0;
    extern __shared__ __align__(16) u32 smem32[];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u32 grp = lane / L, gl = lane % L, gshift = grp * L;
    const u32 gbits = L == 32 ? FULL : (1u << L) - 1u;
    const u32 group_slots = (2u << a.tbits) >> NG_LOG;          // 16-bit slots per group
    unsigned short* tab = reinterpret_cast<unsigned short*>(smem32 + (size_t)warp * (1u << a.tbits)) +
                          (size_t)grp * group_slots;
    const u32 tw_max = a.tbits + 1 - NG_LOG;
    const u64 n_ent = min((u64)*(volatile unsigned long long*)&ctr->entries, a.ent_cap);
    u64 my_steps = 0, my_baby = 0;
    for (;;) {
        u64 first = 0;
        if (lane == 0) first = atomicAdd(&ctr->work_next, (unsigned long long)NG);
        first = __shfl_sync(FULL, first, 0);
        if (first >= n_ent) break;
        const u64 idx = first + grp;
        Entry e = a.ent[idx < n_ent ? idx : n_ent - 1];
        bool active = idx < n_ent;
        // the host sends only p < 2^49 and at most half a group table of baby steps here
        if (active && (e.p >= kFp64Limit || e.m > (1u << (tw_max - 1)))) {
            if (gl == 0) atomicOr(&ctr->status, kStatusBadLaunch);
            active = false;
        }
        Fp64 f;
        f.init(active ? e.p : 1000003ull);
        const u32 m = active ? e.m : 0;
        const u32 jc = active ? (u32)e.jcount : 0;
        const u32 tw = min(tw_max, max(6u, 32u - __clz(max(m, 2u) - 1) + a.load_shift));
        const u32 mask = (1u << tw) - 1, shift = 32 - tw;
        const double B = active ? (double)e.B : 1.0, Bm = active ? (double)e.Bm : 1.0;
        const double tv = active ? (double)e.t : 1.0, G0 = active ? (double)e.G0 : 1.0;

        double xb = B, xg = Bm;                                 // B^(gl+1), Bm^(gl+1)
#pragma unroll
        for (int off = 1; off < L; off <<= 1) {
            const double yb = __shfl_up_sync(FULL, xb, off, L), yg = __shfl_up_sync(FULL, xg, off, L);
            if (gl >= (u32)off) {
                xb = f.mul(xb, yb);
                xg = f.mul(xg, yg);
            }
        }
        const double BL = __shfl_sync(FULL, xb, L - 1, L), BmL = __shfl_sync(FULL, xg, L - 1, L);
        double bl = __shfl_up_sync(FULL, xb, 1, L);
        if (gl == 0) bl = 1.0;
        double Bstep = BL, Gstep = BmL;                         // B^(L CH), Bm^(L CH)
#pragma unroll
        for (int c = 1; c < CH; c <<= 1) {
            Bstep = f.mul(Bstep, Bstep);
            Gstep = f.mul(Gstep, Gstep);
        }
        const double tbl = f.mul(tv, bl);
        double bx[CH], gx[CH];
        bx[0] = tbl;
        gx[0] = f.mul(G0, xg);
#pragma unroll
        for (int c = 1; c < CH; ++c) {
            bx[c] = f.mul(bx[c - 1], BL);
            gx[c] = f.mul(gx[c - 1], BmL);
        }
        uint4* t4 = reinterpret_cast<uint4*>(tab);
        for (u32 k = gl; k <= (mask >> 3); k += L) t4[k] = make_uint4(0, 0, 0, 0);
        __syncwarp();

        // baby steps, each group stopping at its own cycle B^d == 1 (d < m)
        u32 cyc = 0, baby_done = m;
        bool bdone = m == 0;
        const u32 m_max = __reduce_max_sync(FULL, m);
        for (u32 base = 0; base < m_max; base += L * CH) {
            double cv[CH], nb[CH];
            bool hit = false;
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                cv[c] = f.canon(bx[c]);
                nb[c] = f.mul(bx[c], Bstep);               // the next value, independent of the inserts
                hit |= !bdone && base + L * c + gl - 1u < m - 1u && cv[c] == tv;
            }
            u32 cb = 0;
            if (__any_sync(FULL, hit)) {                    // a cycle in some group: locate it exactly
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    const u32 i = base + L * c + gl;
                    const u32 gb = (__ballot_sync(FULL, !bdone && i > 0 && i < m && cv[c] == tv) >> gshift) & gbits;
                    if (gb && !cb) cb = base + L * c + __ffs(gb) - 1;
                }
            }
            const u32 lim = cb ? cb : m;
#pragma unroll
            for (int c = 0; c < CH; ++c)
                if (!bdone && base + L * c + gl < lim) h_insert(tab, mask, shift, hkey_canon(cv[c]));
            if (cb && !bdone) {
                cyc = cb;
                baby_done = cb;
            }
            bdone = bdone || cb != 0 || base + L * CH >= m;
            if (__all_sync(FULL, bdone)) break;
#pragma unroll
            for (int c = 0; c < CH; ++c) bx[c] = nb[c];
        }
        __syncwarp();

        u64 best = ~0ull;
        // a cycle: the j in [1, cyc) with G0 == t B^(cyc - j)
        {
            const int i = gfind_baby<L>(f, tbl, BL, 1, cyc, G0, cyc != 0, gl, gshift, gbits);
            if (cyc && i > 0) best = cyc - (u32)i;
        }
        const u32 G = (active && !cyc && jc > 1) ? (jc - 1 + m - 1) / m : 0;   // g = 1..G covers j in [1, G*m]
        u32 giant_done = G;
        bool gdone = G == 0;
        const u32 G_max = __reduce_max_sync(FULL, G);
        for (u32 base = 0; base < G_max; base += L * CH) {
            u32 hs[CH];
            double nx[CH];
            bool flag = false;
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                hs[c] = hkey_canon(f.canon(gx[c]));
                nx[c] = f.mul(gx[c], Gstep);                   // the next value, independent of the probe
                const u32 slot = tab[hs[c] >> shift];
                flag |= !gdone && ((((slot ^ hfp(hs[c])) & 0x7FFFu) == 0) | ((slot & 0x8000u) != 0));
            }
            if (__any_sync(FULL, flag)) {
                u32 real = 0;
#pragma unroll
                for (int c = 0; c < CH; ++c)
                    if (!gdone && base + L * c + gl + 1 <= G && h_contains(tab, mask, shift, hs[c])) real |= 1u << c;
                u64 jb = ~0ull;
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    u32 gb = (__ballot_sync(FULL, (real >> c) & 1u) >> gshift) & gbits;
                    const double cvc = f.canon(gx[c]);
                    while (__any_sync(FULL, gb != 0 && jb == ~0ull)) {
                        const bool mine = gb != 0 && jb == ~0ull;
                        const int src = mine ? __ffs(gb) - 1 : 0;
                        const double v = __shfl_sync(FULL, cvc, gshift + (u32)src);
                        const int i = gfind_baby<L>(f, tbl, BL, 0, m, v, mine, gl, gshift, gbits);
                        if (mine) {
                            gb &= gb - 1;
                            if (i >= 0) jb = (u64)(base + L * c + (u32)src + 1) * m - (u64)i;
                        }
                    }
                }
                if (jb != ~0ull && !gdone) {
                    best = jb;
                    giant_done = min(G, base + L * CH);
                    gdone = true;
                }
            }
            gdone = gdone || base + L * CH >= G;
            if (__all_sync(FULL, gdone)) break;
#pragma unroll
            for (int c = 0; c < CH; ++c) gx[c] = nx[c];
        }
        __syncwarp();
        if (gl == 0 && active) {
            if (best < e.jcount) emit_relation(e.p, e.n_first + best * e.L, 0, e.item, a.rel, a.rel_cap, ctr);
            my_steps += (u64)baby_done + giant_done;
            my_baby += baby_done;
        }
    }
    if (gl == 0 && my_steps) {
        atomicAdd(&ctr->steps, (unsigned long long)my_steps);
        atomicAdd(&ctr->baby, (unsigned long long)my_baby);
    }
}

// -------------------------------------------------------------- the order --

// y^2 + c in [0, n) (Montgomery squaring; any polynomial map serves rho).
__device__ __forceinline__ u64 rho_step(const Mont& R, u64 y, u64 c) {
    u64 z = R.norm(R.mul(y, y)) + c;
    return z >= R.p ? z - R.p : z;
}

// Pollard-Brent rho with the 32 lanes of a warp walking 32 different maps
// y -> y^2 + c (c = c0 + lane) in lockstep; the first lane whose batch gcd
// gives a nontrivial factor wins (a batch that overshoots to n is replayed
// step by step from its start).  Returns a nontrivial factor of the odd
// composite n < 2^62, or 0 after four rounds of 32 maps.  Warp-uniform.
__device__ u64 warp_rho_factor(u64 n) {
    const u32 lane = threadIdx.x & 31;
    Mont R;
    R.init(n);
    for (u64 c0 = 1; c0 < 1 + 32 * 4; c0 += 32) {
        const u64 c = c0 + lane;
        u64 y = R.one, q = R.one, x = 0, ys = 0, g = 1;
        bool stop = false;
        for (u64 r = 1; r <= (1ull << 24) && !stop; r <<= 1) {
            if (g == 1) x = y;                         // a lane that found g keeps its x and ys for the replay
            for (u64 i = 0; i < r; ++i) y = rho_step(R, y, c);
            for (u64 k = 0; k < r && !stop; k += 128) {
                if (g == 1) ys = y;
                const u64 lim = min((u64)128, r - k);
                for (u64 i = 0; i < lim; ++i) {
                    y = rho_step(R, y, c);
                    q = R.mul(q, x > y ? x - y : y - x);
                }
                if (g == 1) g = gcd64(R.norm(q), n);
                stop = __any_sync(FULL, g != 1 && g != n) || __all_sync(FULL, g != 1);
            }
        }
        if (g == n) {                                  // replay this lane's last batch one step at a time
            g = 1;
            for (u32 it = 0; it < 128 && g == 1; ++it) {
                ys = rho_step(R, ys, c);
                g = gcd64(x > ys ? x - ys : ys - x, n);
            }
        }
        const u32 good = __ballot_sync(FULL, g != 1 && g != n);
        if (good) return __shfl_sync(FULL, g, __ffs(good) - 1);
    }
    return 0;
}

// Exact 12-base Miller-Rabin (Math.hpp:209-251) with the bases spread over
// the lanes of a warp: lane k < 12 tries base k.  Warp-uniform result.
__device__ bool warp_is_prime64(u64 n) {
    const u32 lane = threadIdx.x & 31;
    const u32 bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return false;
    for (int i = 0; i < 12; ++i) {
        if (n == bases[i]) return true;
        if (n % bases[i] == 0) return false;
    }
    bool ok = true;
    if (lane < 12) {
        Mont M;
        M.init(n);
        ok = sprp(M, bases[lane], M.r2());
    }
    return __all_sync(FULL, ok);
}

// q = ord_p(b), b mod p != 0, p prime (Math.hpp:294-310), one warp: the
// lanes split the trial division of p - 1 by the sieving primes (divisibility
// by multiplicative inverses); the cofactor is finished by Miller-Rabin /
// Pollard rho; then each prime factor is stripped from the order.
__device__ u64 warp_mult_order(u64 b, u64 p, const SieveTables& t, bool* failed) {
    const u32 lane = threadIdx.x & 31;
    if (p < 1000) {
        u64 x = b % p, k = 1;
        while (x != 1) {
            x = (x * (b % p)) % p;
            ++k;
        }
        return k;
    }
    u64 f[24];
    int nf = 0;
    const u64 pm1 = p - 1;
    const u64 n0 = pm1 >> (__ffsll((long long)pm1) - 1);    // odd part
    f[nf++] = 2;
    for (u32 base = 0; base < kSievePrimes; base += 32) {
        const u32 k = base + lane;
        const u64 q = k < kSievePrimes ? t.sp[k] : 0;
        const bool live = k < kSievePrimes && q * q <= n0;
        const bool div = live && n0 * t.inv[k] <= t.rcp[k];
        u32 bal = __ballot_sync(FULL, div);
        while (bal) {
            const int src = __ffs(bal) - 1;
            bal &= bal - 1;
            const u64 qf = __shfl_sync(FULL, q, src);
            if (nf < 24) f[nf++] = qf;
        }
        if (!__any_sync(FULL, live)) break;
    }
    // the cofactor of n0 by the small factors found
    u64 c = n0;
    for (int i = 1; i < nf; ++i)
        while (c % f[i] == 0) c /= f[i];
    if (c > 1) {
        u64 stack[8];
        int sp = 0;
        stack[sp++] = c;
        while (sp > 0) {
            const u64 x = stack[--sp];
            if (x == 1) continue;
            if (x < (u64)kSieveMaxPrime * kSieveMaxPrime || warp_is_prime64(x)) {
                bool dup = false;
                for (int i = 0; i < nf; ++i) dup |= f[i] == x;
                if (!dup && nf < 24) f[nf++] = x;
                continue;
            }
            const u64 dv = warp_rho_factor(x);
            if (dv == 0 || sp + 2 > 8) {
                *failed = true;
                return 0;
            }
            stack[sp++] = dv;
            stack[sp++] = x / dv;
        }
    }
    // the order, one prime factor q of p - 1 per lane (nf <= 24): with q^k the
    // power of q in p - 1, x = b^((p-1)/q^k) has order q^j, the q-part of
    // ord_p(b); the order is the product of the lanes' parts
    Mont M;
    M.init(p);
    const u64 bm = M.to_mont(b % p, M.r2());
    u64 q = 0;
#pragma unroll
    for (int i = 0; i < 24; ++i)
        if (i < nf && (u32)i == lane) q = f[i];
    u64 part = 1;
    if (q) {
        u64 t = pm1;
        while (t % q == 0) t /= q;                     // t = (p - 1) / q^k
        u64 x = M.pow(bm, t);
        while (x != M.one) {
            x = M.pow(x, q);
            part *= q;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) part *= __shfl_xor_sync(FULL, part, off);
    return part;
}

// One warp per relation: exact primality of p (composite survivors are
// dropped, q = ~0) and q = ord_p(b).
__global__ void __launch_bounds__(128) k_order(OrderArgs a, Counters* ctr) {
    const u64 n = min((u64)*(volatile unsigned long long*)&ctr->relations, a.rel_cap);
    const u32 lane = threadIdx.x & 31;
    const u64 w0 = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
    const u64 nw = ((u64)gridDim.x * blockDim.x) >> 5;
    for (u64 i = w0; i < n; i += nw) {
        RawRelation r = a.rel[i];
        if (!warp_is_prime64(r.p)) {
            r.q = ~0ull;
        } else if (r.q == 0) {
            const DevItem& it = a.items[r.item];
            const u64 b_mod = residue128(it.babs_hi, it.babs_lo, it.b_neg, r.p);
            bool failed = false;
            r.q = warp_mult_order(b_mod, r.p, a.tables, &failed);
            if (failed && lane == 0) atomicOr(&ctr->status, kStatusOrderFailed);
        }
        if (lane == 0) a.rel[i] = r;
    }
}

// ------------------------------------------------------- served-item state --

// A wave whose buffers overflowed commits nothing: the host redoes its runs
// and records them with k_state_add.
__global__ void k_commit(const WaveDesc* w, const RawRelation* rel, const Counters* ctr, u64 rel_cap, ItemState* st) {
    if (ctr->status & (kStatusSurvivorOverflow | kStatusEntryOverflow | kStatusRelationOverflow)) return;
    const u32 tid = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 n_runs = w->n_runs;
    if (tid < n_runs) {
        const SieveRun& r = w->runs[tid];
        atomicMax(&st[r.item].p_done, (unsigned long long)r.hi);
        atomicAdd(&st[r.item].waves, 1ull);
    }
    const u64 n = min((u64)ctr->relations, rel_cap);
    for (u64 i = tid; i < n; i += (u64)gridDim.x * blockDim.x) {
        const RawRelation r = rel[i];
        if (r.q == ~0ull) continue;                     // a composite survivor
        ItemState& s = st[r.item];
        const u64 k = atomicAdd(&s.n_rel, 1ull);
        if (s.rel_buf && k < s.rel_cap) s.rel_buf[k] = r;
    }
}

// One run redone on the host path: advance the item to hi, append its relations.
__global__ void k_state_add(ItemState* st, u32 item, u64 hi, const RawRelation* rel, u64 n) {
    ItemState& s = st[item];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicMax(&s.p_done, (unsigned long long)hi);
        atomicAdd(&s.waves, 1ull);
    }
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 k = atomicAdd(&s.n_rel, 1ull);
        if (s.rel_buf && k < s.rel_cap) s.rel_buf[k] = rel[i];
    }
}

// ------------------------------------------------------ prime counting --

// Strong probable-prime test of p to base a (a < p) in field F.
template <class F>
__device__ __forceinline__ bool sprp_f(const F& f, u64 p, u64 a) {
    const u64 pm1 = p - 1;
    const int s = __ffsll((long long)pm1) - 1;
    typename F::V x = f.pow(f.from_u64(a), pm1 >> s);
    u64 y = f.residue(x);
    if (y == 1 || y == pm1) return true;
    for (int r = 1; r < s; ++r) {
        x = f.mul(x, x);
        y = f.residue(x);
        if (y == pm1) return true;
        if (y == 1) return false;
    }
    return false;
}

// Exact primality of an odd p > 37 with no factor <= 37: strong tests to the
// 12 bases 2..37 (the set of is_prime64, Math.hpp:209-251), in field F.
template <class F>
__device__ bool is_prime_f(u64 p) {
    const u32 bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    F f;
    f.init(p);
    for (int i = 0; i < 12; ++i)
        if (!sprp_f(f, p, bases[i])) return false;
    return true;
}

__global__ void __launch_bounds__(256) k_count_primes(const u64* surv, u64 surv_cap, Counters* ctr) {
    const u64 n = min((u64)*(volatile unsigned long long*)&ctr->survivors, surv_cap);
    u32 mine = 0;
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 p = surv[i];
        bool prime;
        if (p < 65536ull * 65536ull) {
            prime = true;                               // survivors below 65536^2 are the primes
        } else {
            prime = p < kFp64Limit ? is_prime_f<FieldF>(p) : is_prime_f<FieldM>(p);
        }
        mine += prime ? 1u : 0u;
    }
    const u32 warp_total = __reduce_add_sync(FULL, mine);
    if ((threadIdx.x & 31) == 0 && warp_total) atomicAdd(&ctr->primes, (unsigned long long)warp_total);
}

// ------------------------------------------------------- roofline probes --

// Independent Montgomery multiplies: 8 chains per thread, no memory traffic;
// the arithmetic ceiling of the BSGS step.
__global__ void __launch_bounds__(256) k_mmul_peak(u64 p0, u32 iters, u64* sink) {
    Mont M;
    M.p = p0 | 1;
    M.ninv = Mont::neg_inverse(M.p);
    M.one = 1;
    u64 x[8];
    const u64 y = (0x9E3779B97F4A7C15ull ^ threadIdx.x) % M.p;
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = (blockIdx.x * 8191ull + threadIdx.x * 31ull + k) % M.p;
    for (u32 i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = M.mul(x[k], y);
    }
    u64 acc = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc ^= x[k];
    if (acc == 0x123456789ull) sink[0] = acc;
}

// Independent exact FP64 modular multiplies (p < 2^49): 8 chains per thread.
__global__ void __launch_bounds__(256) k_fmul_peak(u64 p0, u32 iters, u64* sink) {
    Fp64 f;
    f.init(p0 | 1);
    double x[8];
    const double y = (double)((0x9E3779B97F4A7C15ull ^ threadIdx.x) % f.pi);
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = (double)((blockIdx.x * 8191ull + threadIdx.x * 31ull + k) % f.pi);
    for (u32 i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = f.mul(x[k], y);
    }
    double acc = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += x[k];
    if (acc == 123.0) sink[0] = (u64)acc;
}

// Independent 32-bit multiply-adds: 8 chains per thread.
__global__ void __launch_bounds__(256) k_imad_peak(u32 iters, u32* sink) {
    u32 x[8];
    const u32 a = 0x9E3779B1u ^ threadIdx.x, b = 0x85EBCA6Bu + blockIdx.x;
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = threadIdx.x + k;
    for (u32 i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = x[k] * a + b;
    }
    u32 acc = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc ^= x[k];
    if (acc == 0x12345u) sink[0] = acc;
}

// Conflict-free shared-memory atomicOr: lane l of every warp always hits
// bank l of an 8 KB bitmap (the sieve's segment), 8 independent words per
// thread per iteration.
__global__ void __launch_bounds__(256) k_smem_or_peak(u32 iters, u32* sink) {
    __shared__ u32 bits[kSegWords];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (u32 w = threadIdx.x; w < kSegWords; w += blockDim.x) bits[w] = 0;
    __syncthreads();
    for (u32 i = 0; i < iters; ++i) {
#pragma unroll
        for (u32 k = 0; k < 8; ++k) atomicOr(&bits[lane + 32 * ((warp * 8 + k + i) & 63)], 1u << ((i + k) & 31));
    }
    __syncthreads();
    if (bits[threadIdx.x] == 0x12345u) sink[0] = bits[threadIdx.x];
}

// ------------------------------------------------------------- test hooks --

__global__ void k_is_prime(const u64* n, u32* out, u64 count) {
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count; i += (u64)gridDim.x * blockDim.x)
        out[i] = is_prime64(n[i]) ? 1u : 0u;
}

// cases[5i..5i+4] = p, B, G0, t, jcount (plain residues); one warp per case.
__global__ void k_bsgs_direct(const u64* cases, u64* j_out, u64 count, u32 tbits, u32 table_kind) {
    extern __shared__ __align__(16) u32 smem32[];
    const u64 idx = blockIdx.x;
    if (idx >= count) return;
    const u64* c = cases + 5 * idx;
    const u64 p = c[0];
    Entry e;
    e.p = p; e.B = c[1] % p; e.G0 = c[2] % p; e.t = c[3] % p; e.jcount = c[4];
    e.n_first = 0; e.L = 1; e.item = 0;
    u64 result;
    if (e.jcount == 0) {
        result = ~0ull;
    } else if (e.G0 == e.t) {
        result = 0;
    } else if (e.jcount == 1) {
        result = ~0ull;
    } else {
        u32 m = (u32)isqrt_ceil_dev(e.jcount);
        // the table loads of the sieving path
        const u32 cap = min(kMaxBaby, table_kind == 0 || table_kind == 3 ? 1u << (tbits - 1)
                                      : table_kind == 2                    ? 1u << (tbits + 1 - kDefaultLoadShift)
                                                                           : max(1u, (1u << tbits) / 5));
        if (m > cap) m = cap;
        e.m = m;
        Mont M;
        M.init(p);
        const u64 rr = M.r2();
        e.Bm = M.from_mont(M.pow(M.to_mont(e.B, rr), m));
        if (e.p >= kFp64Limit) result = solve_any<0, 0>(e, smem32, tbits, kDefaultLoadShift, kDefaultFill, nullptr);
        else if (table_kind == 0) result = solve_any<2, 0>(e, smem32, tbits, kDefaultLoadShift, kDefaultFill, nullptr);
        else if (table_kind == 2) result = solve_any<2, 2>(e, smem32, tbits, kDefaultLoadShift, kDefaultFill, nullptr);
        else if (table_kind == 3) result = solve_any<2, 3>(e, smem32, tbits, 0, kDefaultFill, nullptr);
        else result = solve_any<2, 1>(e, smem32, tbits, kDefaultLoadShift, kDefaultFill, nullptr);
    }
    if (threadIdx.x == 0) j_out[idx] = result;
}

__global__ void k_order_direct(const u64* bp, u64* q_out, u64 count, SieveTables t) {
    const u64 w0 = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
    const u64 nw = ((u64)gridDim.x * blockDim.x) >> 5;
    for (u64 i = w0; i < count; i += nw) {
        bool failed = false;
        const u64 q = warp_mult_order(bp[2 * i], bp[2 * i + 1], t, &failed);
        if ((threadIdx.x & 31) == 0) q_out[i] = failed ? 0 : q;
    }
}

// -------------------------------------------------------------- launchers --

size_t bsgs_smem_bytes(u32 tbits, u32 warps_per_block, u32 table_kind) {
    const size_t per_warp = (size_t)(4u << tbits);
    return (size_t)warps_per_block * (table_kind == 3 ? per_warp + per_warp / 8 : per_warp);
}

bool valid_seg_words(u32 seg_words) { return seg_words == 1024 || seg_words == 2048 || seg_words == 4096; }

cudaError_t launch_sieve(const SieveArgs& a, const SieveTables& t, u64* surv, u32* surv_item, u64 surv_cap,
                         Counters* ctr, cudaStream_t s, u32 seg_words) {
    if (!valid_seg_words(seg_words)) return cudaErrorInvalidValue;
    const u64 seg_odds = (u64)seg_words * 32;
    const u64 segs = (a.n_odds + seg_odds - 1) / seg_odds;
    if (segs == 0 && !a.include_two) return cudaSuccess;
    const u64 grid = segs == 0 ? 1 : min(segs, (u64)148 * 8);
    if (seg_words == 1024) k_sieve<1024><<<(unsigned)grid, kSieveThreads, 0, s>>>(a, t, surv, surv_item, surv_cap, ctr);
    else if (seg_words == 4096) k_sieve<4096><<<(unsigned)grid, kSieveThreads, 0, s>>>(a, t, surv, surv_item, surv_cap, ctr);
    else k_sieve<2048><<<(unsigned)grid, kSieveThreads, 0, s>>>(a, t, surv, surv_item, surv_cap, ctr);
    return cudaGetLastError();
}

cudaError_t launch_sieve_wave(const WaveDesc* w, const SieveTables& t, u64* surv, u32* surv_item, u64 surv_cap,
                              Counters* ctr, int grid, cudaStream_t s, u32 seg_words) {
    if (!valid_seg_words(seg_words)) return cudaErrorInvalidValue;
    if (seg_words == 1024) k_sieve_wave<1024><<<grid, kSieveThreads, 0, s>>>(w, t, surv, surv_item, surv_cap, ctr);
    else if (seg_words == 4096) k_sieve_wave<4096><<<grid, kSieveThreads, 0, s>>>(w, t, surv, surv_item, surv_cap, ctr);
    else k_sieve_wave<2048><<<grid, kSieveThreads, 0, s>>>(w, t, surv, surv_item, surv_cap, ctr);
    return cudaGetLastError();
}

cudaError_t launch_prep(const PrepArgs& a, Counters* ctr, int grid, cudaStream_t s) {
    k_prep<<<grid, kPrepThreads, 0, s>>>(a, ctr);
    return cudaGetLastError();
}

// Dynamic shared memory limit of every k_bsgs variant on the current device
// (the attribute is per device; set once per size and device, before any
// graph capture, so that a captured launch never needs it).
cudaError_t bsgs_reserve_smem(size_t smem) {
    constexpr int kDevices = 64;
    static std::mutex lock;
    static size_t done[kDevices] = {};
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= kDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(lock);
    if (smem <= done[dev]) return cudaSuccess;
    for (auto kern : {k_bsgs<0, 0>, k_bsgs<1, 0>, k_bsgs<2, 0>, k_bsgs<4, 0>, k_bsgs<1, 1>, k_bsgs<2, 1>,
                      k_bsgs<4, 1>, k_bsgs<1, 2>, k_bsgs<2, 2>, k_bsgs<4, 2>, k_bsgs<1, 3>, k_bsgs<2, 3>,
                      k_bsgs<4, 3>, k_bsgs_groups<8, 1>,
                      k_bsgs_groups<8, 2>, k_bsgs_groups<16, 1>, k_bsgs_groups<16, 2>}) {
        err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
    }
    done[dev] = smem;
    return cudaSuccess;
}

cudaError_t launch_bsgs(const BsgsArgs& a, Counters* ctr, int grid, cudaStream_t s) {
    const size_t smem = bsgs_smem_bytes(a.tbits, a.warps_per_block,
                                        a.max_p >= kFp64Limit || (a.table_kind == 2 && a.lanes != 32) ? 0 : a.table_kind);
    cudaError_t err = bsgs_reserve_smem(smem);
    if (err != cudaSuccess) return err;
    auto go = [&](auto kern) {
        kern<<<grid, a.warps_per_block * 32, smem, s>>>(a, ctr);
        return cudaGetLastError();
    };
    if (a.max_p >= kFp64Limit) return go(k_bsgs<0, 0>);
    if (a.table_kind == 2 && (a.lanes == 8 || a.lanes == 16)) {
        // groups of lanes per prime: FP64 arithmetic only (the caller checked p < 2^49)
        if (a.lanes == 8) return a.chains == 1 ? go(k_bsgs_groups<8, 1>) : go(k_bsgs_groups<8, 2>);
        return a.chains == 1 ? go(k_bsgs_groups<16, 1>) : go(k_bsgs_groups<16, 2>);
    }
    if (a.table_kind == 3) {
        if (a.chains == 4) return go(k_bsgs<4, 3>);
        if (a.chains == 1) return go(k_bsgs<1, 3>);
        return go(k_bsgs<2, 3>);
    }
    if (a.table_kind == 2) {
        if (a.chains == 4) return go(k_bsgs<4, 2>);
        if (a.chains == 1) return go(k_bsgs<1, 2>);
        return go(k_bsgs<2, 2>);
    }
    if (a.table_kind == 1) {
        if (a.chains == 4) return go(k_bsgs<4, 1>);
        if (a.chains == 1) return go(k_bsgs<1, 1>);
        return go(k_bsgs<2, 1>);
    }
    if (a.chains == 4) return go(k_bsgs<4, 0>);
    if (a.chains == 1) return go(k_bsgs<1, 0>);
    return go(k_bsgs<2, 0>);
}

cudaError_t launch_order(const OrderArgs& a, Counters* ctr, int grid, cudaStream_t s) {
    k_order<<<grid, 128, 0, s>>>(a, ctr);
    return cudaGetLastError();
}

cudaError_t launch_commit(const WaveDesc* w, const RawRelation* rel, const Counters* ctr, u64 rel_cap,
                          ItemState* st, cudaStream_t s) {
    k_commit<<<4, 128, 0, s>>>(w, rel, ctr, rel_cap, st);
    return cudaGetLastError();
}

cudaError_t launch_state_add(ItemState* st, u32 item, u64 hi, const RawRelation* rel, u64 n, cudaStream_t s) {
    k_state_add<<<(unsigned)std::min<u64>((n + 255) / 256 + 1, 256), 256, 0, s>>>(st, item, hi, rel, n);
    return cudaGetLastError();
}

cudaError_t launch_count_primes(const u64* surv, u64 surv_cap, Counters* ctr, int grid, cudaStream_t s) {
    k_count_primes<<<grid, 256, 0, s>>>(surv, surv_cap, ctr);
    return cudaGetLastError();
}

cudaError_t launch_mmul_peak(u64 p, u32 iters, int grid, u64* sink, cudaStream_t s) {
    k_mmul_peak<<<grid, 256, 0, s>>>(p, iters, sink);
    return cudaGetLastError();
}

cudaError_t launch_fmul_peak(u64 p, u32 iters, int grid, u64* sink, cudaStream_t s) {
    k_fmul_peak<<<grid, 256, 0, s>>>(p, iters, sink);
    return cudaGetLastError();
}

cudaError_t launch_imad_peak(u32 iters, int grid, u32* sink, cudaStream_t s) {
    k_imad_peak<<<grid, 256, 0, s>>>(iters, sink);
    return cudaGetLastError();
}

cudaError_t launch_smem_or_peak(u32 iters, int grid, u32* sink, cudaStream_t s) {
    k_smem_or_peak<<<grid, 256, 0, s>>>(iters, sink);
    return cudaGetLastError();
}

cudaError_t launch_is_prime(const u64* n, u32* out, u64 count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_is_prime<<<(unsigned)min((count + 127) / 128, (u64)4096), 128, 0, s>>>(n, out, count);
    return cudaGetLastError();
}

cudaError_t launch_bsgs_direct(const u64* cases, u64* j_out, u64 count, u32 tbits, u32 table_kind, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const size_t smem = bsgs_smem_bytes(tbits, 1, table_kind);
    cudaError_t err = cudaFuncSetAttribute(k_bsgs_direct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    k_bsgs_direct<<<(unsigned)count, 32, smem, s>>>(cases, j_out, count, tbits, table_kind);
    return cudaGetLastError();
}

cudaError_t launch_order_direct(const u64* bp, u64* q_out, u64 count, SieveTables t, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_order_direct<<<(unsigned)min((count + 3) / 4, (u64)4096), 128, 0, s>>>(bp, q_out, count, t);
    return cudaGetLastError();
}

}  // namespace mps
