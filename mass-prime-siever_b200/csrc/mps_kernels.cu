// mps_kernels.cu -- the sm_100a kernels of the siever hot path.
//
//   k_sieve  segment sieve of the odd numbers by the odd primes <= 65521,
//            bitmap in shared memory, survivors compacted to global memory
//            (what psieve does, Gpu.hpp:385-455, sized for 148 SMs)
//   k_prep   per survivor: residues of b and -c, quadratic-character filter
//            (Jacobi), base-2 strong test, power-residue split over
//            g = gcd(Q, p - 1) (Gpu.hpp:465-589, Math.hpp:410-433), BSGS set-up
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

namespace mps {

constexpr u32 FULL = 0xFFFFFFFFu;

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

constexpr u32 kSegWords = 2048;               // 8 KB bitmap
constexpr u32 kSegOdds = kSegWords * 32;      // 65,536 odd numbers per segment
constexpr u32 kSieveThreads = 256;
constexpr u32 kWordsPerThread = kSegWords / kSieveThreads;
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

__global__ void __launch_bounds__(kSieveThreads) k_sieve(SieveArgs a, SieveTables t, u64* surv, u32* surv_item,
                                                         u64 cap, Counters* ctr) {
    __shared__ u32 bits[kSegWords];
    __shared__ u32 med_start[kNumMedium];
    __shared__ u32 warp_sum[kSieveThreads / 32];
    __shared__ unsigned long long block_base;
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (blockIdx.x == 0 && tid == 0 && a.include_two) {
        const u64 slot = atomicAdd(&ctr->survivors, 1ull);
        if (slot < cap) {
            surv[slot] = 2;
            if (surv_item) surv_item[slot] = a.item;
        } else {
            atomicOr(&ctr->status, kStatusSurvivorOverflow);
        }
    }

    const u32 n_med = min(a.n_primes, kNumMedium);
    for (u64 seg = blockIdx.x; seg * kSegOdds < a.n_odds; seg += gridDim.x) {
        const u64 base = seg * kSegOdds;
        const u32 len = (u32)min((u64)kSegOdds, a.n_odds - base);
        const u64 v0 = a.lo_odd + 2 * base;

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
            for (u32 w = tid; w < kSegWords; w += kSieveThreads) {
                u32 word = 0;
#pragma unroll
                for (u32 k = 0; k < kNumPattern; ++k) {
                    word |= pat[k] << off[k];
                    int o = (int)off[k] - (int)step[k];
                    if (o < 0) o += (int)qs[k];
                    off[k] = (u32)o;
                }
                bits[w] = word;
            }
        }
        if (tid >= kNumPattern && tid < n_med) med_start[tid] = (u32)min(first_strike(v0, t.sp[tid], t.rcp[tid]), (u64)kSegOdds);
        __syncthreads();
        // the pattern struck 3..31 themselves when they lie in this segment
        if (v0 <= 31 && tid < kNumPattern) {
            const u32 q = t.sp[tid];
            if (q >= v0) {
                const u32 i = (u32)((q - v0) >> 1);
                if (i < len) atomicAnd(&bits[i >> 5], ~(1u << (i & 31)));
            }
        }

        // 2. primes 37..1021: all threads share each prime.
        for (u32 k = kNumPattern; k < n_med; ++k) {
            const u32 q = t.sp[k];
            for (u32 i = med_start[k] + tid * q; i < len; i += kSieveThreads * q)
                atomicOr(&bits[i >> 5], 1u << (i & 31));
        }
        // 3. primes 1031..65521: one thread per prime.
        for (u32 k = kNumMedium + tid; k < a.n_primes; k += kSieveThreads) {
            const u32 q = t.sp[k];
            const u64 j = first_strike(v0, q, t.rcp[k]);
            for (u64 i = j; i < len; i += q) atomicOr(&bits[(u32)i >> 5], 1u << ((u32)i & 31));
        }
        __syncthreads();

        // 4. survivors: contiguous words per thread, block scan, one global atomic.
        const u32 w0 = tid * kWordsPerThread;
        u32 mine = 0;
#pragma unroll
        for (u32 k = 0; k < kWordsPerThread; ++k) {
            const u32 w = w0 + k;
            u32 x = ~bits[w];
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
        if (lane == 31) warp_sum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            u32 ws = lane < kSieveThreads / 32 ? warp_sum[lane] : 0;
            u32 wincl = ws;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                const u32 y = __shfl_up_sync(FULL, wincl, o);
                if (lane >= (u32)o) wincl += y;
            }
            if (lane < kSieveThreads / 32) warp_sum[lane] = wincl - ws;   // exclusive
            if (lane == kSieveThreads / 32 - 1) block_base = atomicAdd(&ctr->survivors, (unsigned long long)wincl);
        }
        __syncthreads();
        u64 pos = block_base + warp_sum[warp] + (incl - mine);
        for (u32 k = 0; k < kWordsPerThread; ++k) {
            const u32 w = w0 + k;
            u32 x = ~bits[w];
            const u32 first = w * 32;
            if (first >= len) x = 0;
            else if (len - first < 32) x &= (1u << (len - first)) - 1u;
            while (x) {
                const u32 b = __ffs(x) - 1;
                x &= x - 1;
                if (pos < cap) {
                    surv[pos] = v0 + 2ull * (first + b);
                    if (surv_item) surv_item[pos] = a.item;
                }
                ++pos;
            }
        }
        if (pos > cap) atomicOr(&ctr->status, kStatusSurvivorOverflow);
        __syncthreads();
    }
}

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

__device__ void prep_one(u64 p, const DevItem& it, const PrepArgs& a, Counters* ctr) {
    const u64 b_mod = residue128(it.babs_hi, it.babs_lo, it.b_neg, p);
    const u64 c_mod = residue128(it.cabs_hi, it.cabs_lo, it.c_neg, p);
    const u64 t = c_mod == 0 ? 0 : p - c_mod;           // -c mod p
    if (b_mod == 0) {                                   // p | b (Math.hpp:383-385, 496-503)
        if (t == 0) emit_relation(p, (u64)it.N0_raw, 1, it.item_index, a.rel, a.rel_cap, ctr);
        return;
    }
    if (p < 1000) {
        small_prime(p, b_mod, t, it, a, ctr);
        return;
    }
    if (t == 0 || !it.has_work) return;                 // Math.hpp:386-396

    // Quadratic character: b^n == t needs (b/p)^n == (t/p).
    const int jb = jacobi(b_mod, p), jt = jacobi(t, p);
    if (jb == 0 || jt == 0) return;                     // a common factor: p is composite
    int par = -1;                                       // forced parity of n, -1: none
    if (jb == 1) {
        if (jt != 1) return;
    } else {
        par = jt == 1 ? 0 : 1;
        if (!(it.cm & 1) && (int)(it.n_start & 1) != par) return;
    }

    Mont M;
    M.init(p);
    if (!sprp2(M)) return;                              // composite survivor
    if (a.full_mr && !is_prime64(p)) return;
    const u64 rr = M.r2();
    const u64 bm = M.to_mont(b_mod, rr), tm = M.to_mont(t, rr);

    // Power-residue split: with g = gcd(Q, p - 1), e = (p - 1) / g,
    // w = b^e and u = t^e are g-th roots of unity and b^n == t forces
    // w^n == u, i.e. n == r (mod d) with d = ord(w), or no solution.
    u32 d = 1, r = 0;
    const u64 pm1 = p - 1;
    const u64 qh = __umul64hi(pm1, it.Q_rcp);
    u32 rem = (u32)(pm1 - qh * it.Q);
    if (rem >= it.Q) rem -= it.Q;
    const u32 g = gcd32(it.Q, rem);
    if (g > 2) {
        const int tz = __ffs(g) - 1;
        const u64 go = g >> tz;
        const u64 e = (pm1 >> tz) * (0 - Mont::neg_inverse(go));   // exact (p - 1) / g
        const u64 u = M.pow(tm, e), w = M.pow(bm, e);
        u64 x = M.one;
        bool found = false;
        d = g;
        for (u32 k = 0; k < g; ++k) {
            if (!found && x == u) {
                r = k;
                found = true;
            }
            x = M.norm(M.mul(x, w));
            if (x == M.one) {
                d = k + 1;
                break;
            }
        }
        if (!found) return;
    } else if (par >= 0) {
        d = 2;
        r = (u32)par;
    }

    // n = n_start + cm*k (in class) with cm*k == r - n_start (mod d).
    const u32 cmd = it.cmQ % d;
    const u32 want = (r + d - it.nsQ % d) % d;
    u32 k0 = 0, acc = 0;
    bool ok = false;
    for (; k0 < d; ++k0) {
        if (acc == want) {
            ok = true;
            break;
        }
        acc += cmd;
        if (acc >= d) acc -= d;
    }
    if (!ok || k0 >= it.K) return;
    const u32 per = d / gcd32(d, cmd);                  // period of k
    u64 jcount = ((u32)it.K - k0 + per - 1) / per;     // K < 2^32 (N1 - N0 <= 10^7)
    if (jcount > p) jcount = p;                         // ord(B) < p (Math.hpp:398-400)
    const u64 L = it.cm * per;
    const u64 n_first = it.n_start + it.cm * k0;

    const u64 G0 = M.pow(bm, n_first);
    if (G0 == tm) {                                     // j = 0
        emit_relation(p, n_first, 0, it.item_index, a.rel, a.rel_cap, ctr);
        return;
    }
    if (jcount <= 1) return;
    const u64 B = M.pow(bm, L);
    u32 m = (u32)isqrt_ceil_dev(jcount);
    if (m > it.max_baby) m = it.max_baby;
    const u64 Bm = M.pow(B, m);

    const u64 slot = atomicAdd(&ctr->entries, 1ull);
    if (slot >= a.ent_cap) {
        atomicOr(&ctr->status, kStatusEntryOverflow);
        return;
    }
    Entry e;
    e.p = p; e.ninv = M.ninv; e.one = M.one; e.t = tm; e.G0 = G0; e.B = B; e.Bm = Bm;
    e.n_first = n_first; e.L = L; e.jcount = jcount; e.m = m; e.item = it.item_index;
    a.ent[slot] = e;
}

__global__ void __launch_bounds__(256) k_prep(PrepArgs a, Counters* ctr) {
    const u64 n = min((u64)*(volatile unsigned long long*)&ctr->survivors, a.surv_cap);
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u32 item = a.surv_item ? a.surv_item[i] : a.item0;
        prep_one(a.surv[i], a.items[item], a, ctr);
    }
}

// --------------------------------------------------------------- the BSGS --

__device__ __forceinline__ u32 table_slot(u64 v, u32 tbits, u32& fp) {
    const u32 lo = (u32)v, hi = (u32)(v >> 32);
    const u32 x = lo ^ (hi * 0x9E3779B1u);
    fp = x & 0xFFFFFu;
    return (x * 0x85EBCA6Bu) >> (32 - tbits);
}

__device__ __forceinline__ void table_insert(u32* tab, u32 mask, u32 tbits, u64 v, u32 i) {
    u32 fp;
    u32 s = table_slot(v, tbits, fp);
    const u32 entry = (fp << kIdxBits) | i;
    while (atomicCAS(&tab[s], kEmptySlot, entry) != kEmptySlot) s = (s + 1) & mask;
}

// t * B^i == v ?  (exact check of a fingerprint match)
__device__ __noinline__ bool verify_baby(const Mont& M, u64 t, u64 B, u32 i, u64 v) {
    return M.norm(M.mul(t, M.pow(B, i))) == v;
}

// Smallest j = g*m - i over the table entries matching v (a giant value of
// step g); ~0u when none matches exactly.
__device__ __forceinline__ u32 table_probe(const u32* tab, u32 mask, u32 tbits, u64 v, u64 g, u32 m,
                                           const Mont& M, u64 t, u64 B) {
    u32 fp;
    u32 s = table_slot(v, tbits, fp);
    u32 best = ~0u;
    for (;;) {
        const u32 e = tab[s];
        if (e == kEmptySlot) break;
        if ((e >> kIdxBits) == fp) {
            const u32 i = e & ((1u << kIdxBits) - 1);
            if (verify_baby(M, t, B, i, v)) {
                const u32 j = (u32)(g * m - i);
                best = min(best, j);
            }
        }
        s = (s + 1) & mask;
    }
    return best;
}

// Solves one entry with the 32 lanes of the calling warp; returns the
// smallest j (< jcount) or ~0ull.  Two interleaved chains per lane: baby
// indices i = l + 64k and l + 32 + 64k, giant steps g = 1 + l + 64k and
// 33 + l + 64k.
__device__ u64 solve_entry(const Entry& e, u32* tab, u32 tbits, u64* steps_out = nullptr) {
    const u32 lane = threadIdx.x & 31;
    Mont M;
    M.p = e.p; M.ninv = e.ninv; M.one = e.one;
    const u32 m = e.m;
    const u32 T = 1u << tbits, mask = T - 1;

    // lane powers by an inclusive scan: xb = B^(l+1), xg = Bm^(l+1)
    u64 xb = e.B, xg = e.Bm;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const u64 yb = __shfl_up_sync(FULL, xb, off), yg = __shfl_up_sync(FULL, xg, off);
        if (lane >= (u32)off) {
            xb = M.mul(xb, yb);
            xg = M.mul(xg, yg);
        }
    }
    const u64 B32 = __shfl_sync(FULL, xb, 31), Bm32 = __shfl_sync(FULL, xg, 31);
    u64 bl = __shfl_up_sync(FULL, xb, 1);
    if (lane == 0) bl = M.one;                          // B^l
    const u64 B64 = M.mul(B32, B32), Bm64 = M.mul(Bm32, Bm32);
    u64 baby0 = M.mul(e.t, bl), baby1 = M.mul(baby0, B32);
    u64 gi0 = M.mul(e.G0, xg), gi1 = M.mul(gi0, Bm32);

    uint4* t4 = reinterpret_cast<uint4*>(tab);
    for (u32 k = lane; k < T / 4; k += 32) t4[k] = make_uint4(kEmptySlot, kEmptySlot, kEmptySlot, kEmptySlot);
    __syncwarp();

    // baby steps t*B^i, stopping at a cycle B^d == 1 (d < m)
    u32 cyc = 0;
    u64 steps = 0;
    for (u32 base = 0; base < m; base += 64) {
        const u32 i0 = base + lane, i1 = base + 32 + lane;
        const u64 v0 = M.norm(baby0), v1 = M.norm(baby1);
        const u32 b0 = __ballot_sync(FULL, i0 > 0 && i0 < m && v0 == e.t);
        const u32 b1 = __ballot_sync(FULL, i1 < m && v1 == e.t);
        u32 lim = m;
        if (b0 | b1) {
            cyc = b0 ? base + __ffs(b0) - 1 : base + 32 + __ffs(b1) - 1;
            lim = cyc;
        }
        if (i0 < lim) table_insert(tab, mask, tbits, v0, i0);
        if (i1 < lim) table_insert(tab, mask, tbits, v1, i1);
        steps += min(64u, lim - base);
        if (cyc) break;
        baby0 = M.mul(baby0, B64);
        baby1 = M.mul(baby1, B64);
    }
    __syncwarp();

    u64 best = ~0ull;
    if (cyc) {
        // ord(B) = cyc < m: the answer is the j in [1, cyc) with G0 == t*B^(cyc-j)
        // (j = 0 was ruled out by the prep); t*B^i, i < cyc, are distinct.
        u32 jl = ~0u;
        if (lane == 0) {
            u32 fp;
            u32 s = table_slot(e.G0, tbits, fp);
            for (;;) {
                const u32 en = tab[s];
                if (en == kEmptySlot) break;
                const u32 i = en & ((1u << kIdxBits) - 1);
                if ((en >> kIdxBits) == fp && i >= 1 && i < cyc && verify_baby(M, e.t, e.B, i, e.G0))
                    jl = min(jl, cyc - i);
                s = (s + 1) & mask;
            }
        }
        jl = __shfl_sync(FULL, jl, 0);
        if (jl != ~0u) best = jl;
    } else {
        const u64 G = (e.jcount - 1 + m - 1) / m;      // giant steps g = 1..G cover j in [1, G*m]
        for (u64 base = 0; base < G; base += 64) {
            const u64 g0 = base + 1 + lane, g1 = base + 33 + lane;
            u32 cand = ~0u;
            if (g0 <= G) cand = min(cand, table_probe(tab, mask, tbits, M.norm(gi0), g0, m, M, e.t, e.B));
            if (g1 <= G) cand = min(cand, table_probe(tab, mask, tbits, M.norm(gi1), g1, m, M, e.t, e.B));
            const u32 jmin = __reduce_min_sync(FULL, cand);
            steps += min((u64)64, G - base);
            if (jmin != ~0u) {
                best = jmin;
                break;
            }
            gi0 = M.mul(gi0, Bm64);
            gi1 = M.mul(gi1, Bm64);
        }
    }
    __syncwarp();
    if (steps_out) *steps_out = steps;
    return best < e.jcount ? best : ~0ull;
}

__global__ void k_bsgs(BsgsArgs a, Counters* ctr) {
    extern __shared__ __align__(16) u32 smem[];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32* tab = smem + (size_t)warp * (1u << a.tbits);
    const u64 n_ent = min((u64)*(volatile unsigned long long*)&ctr->entries, a.ent_cap);
    u64 my_steps = 0;
    if (a.persistent) {
        for (;;) {
            u64 idx = 0;
            if (lane == 0) idx = atomicAdd(&ctr->work_next, 1ull);
            idx = __shfl_sync(FULL, idx, 0);
            if (idx >= n_ent) break;
            const Entry e = a.ent[idx];
            u64 steps = 0;
            const u64 j = solve_entry(e, tab, a.tbits, &steps);
            if (lane == 0) {
                if (j != ~0ull) emit_relation(e.p, e.n_first + j * e.L, 0, e.item, a.rel, a.rel_cap, ctr);
                my_steps += steps;
            }
        }
        if (lane == 0 && my_steps) atomicAdd(&ctr->steps, (unsigned long long)my_steps);
    } else {
        const u64 idx = (u64)blockIdx.x * a.warps_per_block + warp;
        if (idx >= n_ent) return;
        const Entry e = a.ent[idx];
        u64 steps = 0;
        const u64 j = solve_entry(e, tab, a.tbits, &steps);
        if (lane == 0) {
            if (j != ~0ull) emit_relation(e.p, e.n_first + j * e.L, 0, e.item, a.rel, a.rel_cap, ctr);
            atomicAdd(&ctr->steps, (unsigned long long)steps);
        }
    }
}

// -------------------------------------------------------------- the order --

// y^2 + c in [0, n) (Montgomery squaring; any polynomial map serves rho).
__device__ __forceinline__ u64 rho_step(const Mont& R, u64 y, u64 c) {
    u64 z = R.norm(R.mul(y, y)) + c;
    return z >= R.p ? z - R.p : z;
}

// Pollard-Brent rho on an odd composite n < 2^62 (Montgomery steps); returns
// a nontrivial factor, or 0 after a bounded number of tries.
__device__ u64 rho_factor(u64 n) {
    Mont R;
    R.init(n);
    for (u64 c = 1; c < 64; ++c) {
        u64 y = R.one, q = R.one, g = 1, x = 0, ys = 0;
        u64 r = 1;
        const u64 step_cap = 1ull << 24;
        while (g == 1 && r <= step_cap) {
            x = y;
            for (u64 i = 0; i < r; ++i) y = rho_step(R, y, c);
            for (u64 k = 0; k < r && g == 1; k += 128) {
                ys = y;
                const u64 lim = min((u64)128, r - k);
                for (u64 i = 0; i < lim; ++i) {
                    y = rho_step(R, y, c);
                    q = R.mul(q, x > y ? x - y : y - x);
                }
                g = gcd64(R.norm(q), n);
            }
            r <<= 1;
        }
        if (g == n) {
            g = 1;
            for (u64 it = 0; it < (1ull << 26) && g == 1; ++it) {
                ys = rho_step(R, ys, c);
                g = gcd64(x > ys ? x - ys : ys - x, n);
            }
        }
        if (g != 1 && g != n) return g;
    }
    return 0;
}

// q = ord_p(b), b mod p != 0, p prime (Math.hpp:294-310): factor p - 1 by
// the sieving primes (divisibility by multiplicative inverses), finish the
// cofactor by Miller-Rabin / Pollard rho, then strip each prime factor.
__device__ u64 mult_order(u64 b, u64 p, const SieveTables& t, bool* failed) {
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
    u64 n = p - 1;
    const int tz = __ffsll((long long)n) - 1;
    n >>= tz;
    f[nf++] = 2;
    for (u32 k = 0; k < kSievePrimes; ++k) {
        const u64 q = t.sp[k];
        if (q * q > n) break;
        const u64 qi = t.inv[k], lim = t.rcp[k];
        if (n * qi <= lim) {
            f[nf++] = q;
            do n *= qi; while (n * qi <= lim);
        }
    }
    if (n > 1) {
        u64 stack[8];
        int sp = 0;
        stack[sp++] = n;
        while (sp > 0) {
            const u64 x = stack[--sp];
            if (x == 1) continue;
            if ((x < (u64)kSieveMaxPrime * kSieveMaxPrime) || is_prime64(x)) {
                bool dup = false;
                for (int i = 0; i < nf; ++i) dup |= f[i] == x;
                if (!dup && nf < 24) f[nf++] = x;
                continue;
            }
            const u64 dv = rho_factor(x);
            if (dv == 0 || sp + 2 > 8) {
                *failed = true;
                return 0;
            }
            stack[sp++] = dv;
            stack[sp++] = x / dv;
        }
    }
    Mont M;
    M.init(p);
    const u64 bm = M.to_mont(b % p, M.r2());
    u64 order = p - 1;
    for (int i = 0; i < nf; ++i) {
        while (order % f[i] == 0 && M.pow(bm, order / f[i]) == M.one) order /= f[i];
    }
    return order;
}

__global__ void __launch_bounds__(128) k_order(OrderArgs a, Counters* ctr) {
    const u64 n = min((u64)*(volatile unsigned long long*)&ctr->relations, a.rel_cap);
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        RawRelation r = a.rel[i];
        if (!is_prime64(r.p)) {
            r.q = ~0ull;                                // a composite survivor: dropped
        } else if (r.q == 0) {
            const DevItem& it = a.items[r.item];
            const u64 b_mod = residue128(it.babs_hi, it.babs_lo, it.b_neg, r.p);
            bool failed = false;
            r.q = mult_order(b_mod, r.p, a.tables, &failed);
            if (failed) atomicOr(&ctr->status, kStatusOrderFailed);
        }
        a.rel[i] = r;
    }
}

// ------------------------------------------------------ prime counting --

__global__ void __launch_bounds__(256) k_count_primes(const u64* surv, u64 surv_cap, Counters* ctr) {
    const u64 n = min((u64)*(volatile unsigned long long*)&ctr->survivors, surv_cap);
    u32 mine = 0;
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 p = surv[i];
        bool prime;
        if (p < 1000) {
            prime = true;                               // survivors below 65536^2 are the primes
        } else {
            Mont M;
            M.init(p);
            prime = sprp2(M) && is_prime64(p);
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

// ------------------------------------------------------------- test hooks --

__global__ void k_is_prime(const u64* n, u32* out, u64 count) {
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count; i += (u64)gridDim.x * blockDim.x)
        out[i] = is_prime64(n[i]) ? 1u : 0u;
}

// cases[5i..5i+4] = p, B, G0, t, jcount (plain residues); one warp per case.
__global__ void k_bsgs_direct(const u64* cases, u64* j_out, u64 count, u32 tbits) {
    extern __shared__ __align__(16) u32 smem[];
    const u64 idx = blockIdx.x;
    if (idx >= count) return;
    const u64* c = cases + 5 * idx;
    Mont M;
    M.init(c[0]);
    const u64 rr = M.r2();
    Entry e;
    e.p = c[0]; e.ninv = M.ninv; e.one = M.one;
    e.B = M.to_mont(c[1] % c[0], rr);
    e.G0 = M.to_mont(c[2] % c[0], rr);
    e.t = M.to_mont(c[3] % c[0], rr);
    e.jcount = c[4];
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
        const u32 cap = min(kMaxBaby, (1u << tbits) / 2);
        if (m > cap) m = cap;
        e.m = m;
        e.Bm = M.pow(e.B, m);
        result = solve_entry(e, smem, tbits);
    }
    if (threadIdx.x == 0) j_out[idx] = result;
}

__global__ void k_order_direct(const u64* bp, u64* q_out, u64 count, SieveTables t) {
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count; i += (u64)gridDim.x * blockDim.x) {
        bool failed = false;
        const u64 q = mult_order(bp[2 * i], bp[2 * i + 1], t, &failed);
        q_out[i] = failed ? 0 : q;
    }
}

// -------------------------------------------------------------- launchers --

size_t bsgs_smem_bytes(u32 tbits, u32 warps_per_block) { return (size_t)warps_per_block * (4u << tbits); }

cudaError_t launch_sieve(const SieveArgs& a, const SieveTables& t, u64* surv, u32* surv_item, u64 surv_cap,
                         Counters* ctr, cudaStream_t s) {
    const u64 segs = (a.n_odds + kSegOdds - 1) / kSegOdds;
    if (segs == 0 && !a.include_two) return cudaSuccess;
    const u64 grid = segs == 0 ? 1 : min(segs, (u64)148 * 8);
    k_sieve<<<(unsigned)grid, kSieveThreads, 0, s>>>(a, t, surv, surv_item, surv_cap, ctr);
    return cudaGetLastError();
}

cudaError_t launch_prep(const PrepArgs& a, Counters* ctr, int grid, cudaStream_t s) {
    k_prep<<<grid, 256, 0, s>>>(a, ctr);
    return cudaGetLastError();
}

cudaError_t launch_bsgs(const BsgsArgs& a, Counters* ctr, int grid, cudaStream_t s) {
    const size_t smem = bsgs_smem_bytes(a.tbits, a.warps_per_block);
    cudaError_t err = cudaFuncSetAttribute(k_bsgs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    k_bsgs<<<grid, a.warps_per_block * 32, smem, s>>>(a, ctr);
    return cudaGetLastError();
}

cudaError_t launch_order(const OrderArgs& a, Counters* ctr, int grid, cudaStream_t s) {
    k_order<<<grid, 128, 0, s>>>(a, ctr);
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

cudaError_t launch_imad_peak(u32 iters, int grid, u32* sink, cudaStream_t s) {
    k_imad_peak<<<grid, 256, 0, s>>>(iters, sink);
    return cudaGetLastError();
}

cudaError_t launch_is_prime(const u64* n, u32* out, u64 count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_is_prime<<<(unsigned)min((count + 127) / 128, (u64)4096), 128, 0, s>>>(n, out, count);
    return cudaGetLastError();
}

cudaError_t launch_bsgs_direct(const u64* cases, u64* j_out, u64 count, u32 tbits, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const size_t smem = (size_t)4 << tbits;
    cudaError_t err = cudaFuncSetAttribute(k_bsgs_direct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    k_bsgs_direct<<<(unsigned)count, 32, smem, s>>>(cases, j_out, count, tbits);
    return cudaGetLastError();
}

cudaError_t launch_order_direct(const u64* bp, u64* q_out, u64 count, SieveTables t, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_order_direct<<<(unsigned)min((count + 63) / 64, (u64)4096), 64, 0, s>>>(bp, q_out, count, t);
    return cudaGetLastError();
}

}  // namespace mps
