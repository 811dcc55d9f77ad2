// arith.cuh -- exact 64-bit modular arithmetic for the sm_100a kernels.
//
// Montgomery multiplication modulo an odd p < 2^62 with R = 2^64, written
// for the integer multiply pipe: one 64x64->128 product, one 64-bit low
// product and one high product per multiply.  Values are kept "lazy" in
// [0, 2p): for a, b < 2p and p < 2^62, (a*b + m*p) / R < 2p, so no final
// subtraction is needed between multiplies; norm() brings a value to [0, p)
// where it is compared or hashed.  Same arithmetic as the reference's
// Montgomery (Math.hpp:29-79) and mmul/mpow (Gpu.hpp:77-96), restated.
#pragma once

#include "mps_common.cuh"

namespace mps {

struct Mont {
    u64 p;      // odd modulus, p < 2^62
    u64 ninv;   // -p^-1 mod 2^64
    u64 one;    // R mod p (the Montgomery form of 1)

    // Newton iteration for p^-1 mod 2^64: 3p xor 2 is correct to 5 bits,
    // each step doubles the correct bits (5 -> 10 -> 20 -> 40 -> 80).
    __device__ __forceinline__ static u64 neg_inverse(u64 p) {
        u64 inv = (3 * p) ^ 2;
        inv *= 2 - p * inv;
        inv *= 2 - p * inv;
        inv *= 2 - p * inv;
        inv *= 2 - p * inv;
        return 0 - inv;
    }

    __device__ __forceinline__ void init(u64 modulus) {
        p = modulus;
        ninv = neg_inverse(modulus);
        one = (0 - modulus) % modulus;
    }

    __device__ __forceinline__ u64 mul(u64 a, u64 b) const {
        const u64 lo = a * b;
        const u64 hi = __umul64hi(a, b);
        const u64 m = lo * ninv;
        const u64 mh = __umul64hi(m, p);
        // lo + (m*p mod 2^64) is 0 (lo == 0) or exactly 2^64 (carry 1).
        return hi + mh + (lo != 0 ? 1ull : 0ull);
    }

    __device__ __forceinline__ u64 norm(u64 a) const { return a >= p ? a - p : a; }

    // 2a for a lazy value a < 2p, kept below 2p.
    __device__ __forceinline__ u64 dbl(u64 a) const {
        u64 x = a + a;
        return x >= 2 * p ? x - 2 * p : x;
    }

    // R^2 mod p from R mod p: four doublings give 16R, four Montgomery
    // squarings give 2^8 R, 2^16 R, 2^32 R, 2^64 R = R^2.
    __device__ __forceinline__ u64 r2() const {
        u64 a = one;
        a = dbl(a); a = dbl(a); a = dbl(a); a = dbl(a);
        a = mul(a, a); a = mul(a, a); a = mul(a, a); a = mul(a, a);
        return norm(a);
    }

    __device__ __forceinline__ u64 to_mont(u64 a, u64 rr) const { return norm(mul(a, rr)); }
    __device__ __forceinline__ u64 from_mont(u64 a) const { return norm(mul(a, 1)); }

    // base^e (Montgomery form in and out, result normalised).
    __device__ __forceinline__ u64 pow(u64 base, u64 e) const {
        u64 r = one;
        while (e) {
            if (e & 1) r = mul(r, base);
            base = mul(base, base);
            e >>= 1;
        }
        return norm(r);
    }
};

__device__ __forceinline__ u64 gcd64(u64 a, u64 b) {
    while (b) {
        const u64 t = a % b;
        a = b;
        b = t;
    }
    return a;
}

__device__ __forceinline__ u32 gcd32(u32 a, u32 b) {
    while (b) {
        const u32 t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// a^-1 mod m for gcd(a, m) = 1, 0 <= a < m (extended Euclid; m == 1 gives 0).
__device__ __forceinline__ u32 inv_mod32(u32 a, u32 m) {
    u32 r0 = m, r1 = a;
    long long s0 = 0, s1 = 1;                          // |s| <= m
    while (r1) {
        const u32 q = r0 / r1, r2 = r0 - q * r1;
        const long long s2 = s0 - (long long)q * s1;
        r0 = r1; r1 = r2; s0 = s1; s1 = s2;
    }
    return (u32)(s0 < 0 ? s0 + m : s0) % m;
}

// Jacobi symbol (a/n) for odd n < 2^32, a < n: the binary algorithm (strip
// twos with (2/n) = -1 iff n == 3, 5 mod 8; swap with reciprocity, sign -1
// iff both are 3 mod 4).  Returns 1, -1, or 0 when gcd(a, n) > 1.
__device__ __forceinline__ int jacobi32(u32 a, u32 n) {
    u32 neg = 0;
    while (a != 0) {
        const int tz = __ffs((int)a) - 1;
        a >>= tz;
        if ((tz & 1) && ((n & 7u) == 3u || (n & 7u) == 5u)) neg ^= 1u;
        if (a < n) {
            const u32 x = a;
            a = n;
            n = x;
            if ((a & n & 3u) == 3u) neg ^= 1u;
        }
        a -= n;
    }
    return n == 1 ? (neg ? -1 : 1) : 0;
}

// x mod o for an odd o < 2^32 from rcp = floor((2^64 - 1) / o).
__device__ __forceinline__ u32 mod_small(u64 x, u32 o, u64 rcp) {
    const u64 q = __umul64hi(x, rcp);
    u64 r = x - q * o;
    if (r >= o) r -= o;
    return (u32)r;
}

// The Jacobi symbol (x/p) for odd p > o and x = (-1)^neg 2^k o, o odd:
// (-1/p) = -1 iff p == 3 mod 4, (2/p) = -1 iff p == 3, 5 mod 8, and by
// reciprocity (o/p) = (p mod o / o), negated iff o and p are both 3 mod 4.
// 0 when gcd(o, p) > 1.
__device__ __forceinline__ int jacobi_small(u64 p, u32 neg, u32 k, u32 o, u64 rcp) {
    const u32 p8 = (u32)p & 7u;
    u32 flip = 0;
    if (neg && (p8 & 3u) == 3u) flip ^= 1u;
    if ((k & 1u) && (p8 == 3u || p8 == 5u)) flip ^= 1u;
    int j = 1;
    if (o > 1) {
        j = jacobi32(mod_small(p, o, rcp), o);
        if ((o & 3u) == 3u && (p8 & 3u) == 3u) flip ^= 1u;
    }
    return flip ? -j : j;
}

// Strong test to base a (a < p), Montgomery form.
__device__ __forceinline__ bool sprp(const Mont& M, u64 a, u64 rr) {
    const u64 pm1 = M.p - 1;
    const int s = __ffsll((long long)pm1) - 1;
    const u64 d = pm1 >> s;
    const u64 minus_one = M.p - M.one;
    u64 x = M.pow(M.to_mont(a, rr), d);
    if (x == M.one || x == minus_one) return true;
    for (int r = 1; r < s; ++r) {
        x = M.norm(M.mul(x, x));
        if (x == minus_one) return true;
        if (x == M.one) return false;
    }
    return false;
}

// Exact deterministic primality for n < 2^62 (Math.hpp:209-251): trial
// division by the 12 bases, then strong tests to the same 12 bases.
__device__ __noinline__ bool is_prime64(u64 n) {
    const u32 bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return false;
    for (int i = 0; i < 12; ++i) {
        if (n == bases[i]) return true;
        if (n % bases[i] == 0) return false;
    }
    Mont M;
    M.init(n);
    const u64 rr = M.r2();
    for (int i = 0; i < 12; ++i)
        if (!sprp(M, bases[i], rr)) return false;
    return true;
}

// Exact modular multiplication on the FP64 pipe for odd p < 2^49.
//
// Values are doubles holding integers; "lazy" values lie in (-2p, 2p) and a
// product lands in (-p, p).  For |a|, |b| < 2p < 2^50:
//   h = fl(a*b), l = fma(a, b, -h)          a*b = h + l exactly (|l| <= 2^46)
//   q = nearest integer to h * fl(1/p)      via fma(h, pinv, 1.5*2^52) - 1.5*2^52
//   r = fma(-q, p, h)                       exact: h - q*p is an integer, |.| <= 0.75p
//   r + l                                   exact, == a*b (mod p), |.| <= p
// (|h*pinv| < 2^51 keeps the rounding trick exact.)  Every operation uses an
// explicit round-to-nearest intrinsic so that nothing is contracted or
// reassociated.  A zero product never occurs in the solve (all values are
// units), so |r + l| < p there and one conditional +p gives [0, p).
struct Fp64 {
    double p, pinv;
    u64 pi;

    __device__ __forceinline__ void init(u64 modulus) {
        pi = modulus;
        p = (double)modulus;
        pinv = __drcp_rn(p);                   // correctly rounded 1/p (the value 1.0 / p gives)
    }
    __device__ __forceinline__ double mul(double a, double b) const {
        const double C = 6755399441055744.0;   // 1.5 * 2^52
        const double h = __dmul_rn(a, b);
        const double l = __fma_rn(a, b, -h);
        const double q = __dsub_rn(__fma_rn(h, pinv, C), C);
        const double r = __fma_rn(-q, p, h);
        return __dadd_rn(r, l);
    }
    // [0, p) representative of a value in (-p, p).
    __device__ __forceinline__ double canon(double a) const {
        if (a < 0.0) a = __dadd_rn(a, p);
        return a;
    }
    // The integer of a canonical value (exact: a + 2^52 < 2^53).
    __device__ __forceinline__ u64 bits(double a) const {
        return (u64)__double_as_longlong(__dadd_rn(a, 4503599627370496.0)) & ((1ull << 52) - 1);
    }
    __device__ __forceinline__ double from_u64(u64 x) const { return (double)x; }   // x < p < 2^49: exact
    __device__ __forceinline__ double one() const { return 1.0; }
    // Exact [0, p) residue of any lazy value in (-2p, 2p) (prep paths, zero allowed).
    __device__ __forceinline__ u64 residue(double a) const {
        double x = a;
        if (x < 0.0) x = __dadd_rn(x, p);
        if (x < 0.0) x = __dadd_rn(x, p);
        if (x >= p) x = __dsub_rn(x, p);
        return (u64)x;
    }
    __device__ __forceinline__ double pow(double base, u64 e) const {
        double r = 1.0;
        while (e) {
            if (e & 1) r = mul(r, base);
            base = mul(base, base);
            e >>= 1;
        }
        return r;
    }
};

// Plain modular product for moduli below 2^32 (small-prime paths).
__device__ __forceinline__ u64 mulmod_small(u64 a, u64 b, u64 p) { return (a * b) % p; }

}  // namespace mps
