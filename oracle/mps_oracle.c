/*
 * mps_oracle.c -- CPU restatement of the Mass Prime Siever 14.0 hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): the sieve,
 * the 12-base Miller-Rabin, the Montgomery arithmetic, the exact BSGS of
 * run_bsgs, and the multiplicative order, each restated in plain C from the
 * reference function it cites.  References are "Mass Prime Siever/<file>:<line>".
 *
 * One deliberate difference: the order q = ord_p(b) (Math.hpp:294-310)
 * factors p - 1 with Pollard-Brent rho seeded by a fixed sequence instead
 * of std::mt19937_64.  The order of b modulo p does not depend on how p - 1
 * is factored, so q is identical.
 */
#include "mps_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;
typedef __int128 i128;

/* ---- work counters (thread-local; only the counted entry point reads them) ---- */
static __thread uint64_t tl_mul;

/* Math.hpp:22-26 */
static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t n) {
    ++tl_mul;
    return (uint64_t)(((u128)(a % n) * (b % n)) % n);
}

/* Math.hpp:126-140 */
uint64_t mpo_powmod(uint64_t a, uint64_t e, uint64_t n) {
    if (n == 1) return 0;
    uint64_t r = 1;
    a %= n;
    while (e) {
        if (e & 1) r = mulmod(r, a, n);
        a = mulmod(a, a, n);
        e >>= 1;
    }
    return r;
}

/* Math.hpp:209-251: trial division by the 12 bases, then strong tests to
 * the same 12 bases (exact for every 64-bit n). */
int mpo_is_prime64(uint64_t n) {
    static const uint64_t bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; ++i) {
        if (n == bases[i]) return 1;
        if (n % bases[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; ++s; }
    for (int i = 0; i < 12; ++i) {
        uint64_t x = mpo_powmod(bases[i] % n, d, n);
        if (x == 1 || x == n - 1) continue;
        int ok = 0;
        for (int r = 1; r < s; ++r) {
            x = mulmod(x, x, n);
            if (x == n - 1) { ok = 1; break; }
        }
        if (!ok) return 0;
    }
    return 1;
}

/* Gpu.hpp:213-226: binary Jacobi symbol, n odd. */
int mpo_jacobi(uint64_t a, uint64_t n) {
    int s = 1;
    while (a != 0) {
        const int flip2 = ((n & 7) == 3 || (n & 7) == 5);
        while ((a & 1) == 0) { a >>= 1; if (flip2) s = -s; }
        if (a < n) {
            const uint64_t x = a; a = n; n = x;
            if ((a & 3) == 3 && (n & 3) == 3) s = -s;
        }
        a -= n;
    }
    return n == 1 ? s : 0;
}

/* ---- Montgomery arithmetic, Math.hpp:29-79 ---- */
typedef struct mont { uint64_t n, ninv, one, r2; } mont;

static void mont_init(mont* m, uint64_t n) {
    uint64_t inv = n;                 /* 3 correct bits for odd n; 5 Newton steps -> 96 */
    for (int i = 0; i < 5; ++i) inv *= 2 - n * inv;
    m->n = n;
    m->ninv = 0 - inv;
    m->one = (0 - n) % n;
    m->r2 = (uint64_t)(((u128)m->one * m->one) % n);
}

static uint64_t mont_redc(const mont* m, uint64_t hi, uint64_t lo) {
    const uint64_t q = lo * m->ninv;
    const u128 qn = (u128)q * m->n;
    const u128 s = (u128)lo + (uint64_t)qn;          /* low word is 0, keeps the carry */
    const uint64_t t = hi + (uint64_t)(qn >> 64) + (uint64_t)(s >> 64);
    return t >= m->n ? t - m->n : t;
}

static uint64_t mont_mul(const mont* m, uint64_t a, uint64_t b) {
    ++tl_mul;
    const u128 x = (u128)a * b;
    return mont_redc(m, (uint64_t)(x >> 64), (uint64_t)x);
}

static uint64_t mont_to(const mont* m, uint64_t a) { return mont_mul(m, a % m->n, m->r2); }

static uint64_t mont_pow(const mont* m, uint64_t base, uint64_t e) {
    uint64_t r = m->one;
    while (e) {
        if (e & 1) r = mont_mul(m, r, base);
        base = mont_mul(m, base, base);
        e >>= 1;
    }
    return r;
}

static int mont_legendre(const mont* m, uint64_t a) {
    if (a == 0) return 0;
    return mont_pow(m, a, (m->n - 1) >> 1) == m->one ? 1 : -1;
}

void mpo_mont_consts(uint64_t n, uint64_t* ninv, uint64_t* one, uint64_t* r2) {
    mont m;
    mont_init(&m, n);
    *ninv = m.ninv; *one = m.one; *r2 = m.r2;
}

uint64_t mpo_mont_mul(uint64_t a, uint64_t b, uint64_t n, uint64_t ninv) {
    mont m = {n, ninv, 0, 0};
    return mont_mul(&m, a, b);
}

/* ---- flat open-addressing table, Math.hpp:82-124 (insert keeps the first index) ---- */
typedef struct baby_table {
    uint64_t* keys;
    uint32_t* vals;
    uint64_t cap;
    unsigned bits;
} baby_table;
static __thread baby_table tl_table;
#define EMPTY_KEY (~0ULL)

static void table_reset(baby_table* t, uint64_t entries) {
    unsigned bits = 4;
    while ((1ULL << bits) < entries * 2) ++bits;
    t->bits = bits;
    const uint64_t size = 1ULL << bits;
    if (t->cap < size) {
        free(t->keys); free(t->vals);
        t->keys = (uint64_t*)malloc(size * sizeof(uint64_t));
        t->vals = (uint32_t*)malloc(size * sizeof(uint32_t));
        t->cap = size;
    }
    memset(t->keys, 0xFF, size * sizeof(uint64_t));
}

static uint64_t table_slot(const baby_table* t, uint64_t key) {
    return (key * 0x9E3779B97F4A7C15ULL) >> (64 - t->bits);
}

static void table_insert(baby_table* t, uint64_t key, uint32_t val) {
    const uint64_t mask = (1ULL << t->bits) - 1;
    uint64_t h = table_slot(t, key);
    while (t->keys[h] != EMPTY_KEY) {
        if (t->keys[h] == key) return;
        h = (h + 1) & mask;
    }
    t->keys[h] = key;
    t->vals[h] = val;
}

static int table_find(const baby_table* t, uint64_t key, uint32_t* val) {
    const uint64_t mask = (1ULL << t->bits) - 1;
    uint64_t h = table_slot(t, key);
    while (t->keys[h] != EMPTY_KEY) {
        if (t->keys[h] == key) { *val = t->vals[h]; return 1; }
        h = (h + 1) & mask;
    }
    return 0;
}

/* ---- integer helpers, Math.hpp:146-207 ---- */
static i128 item_b(const mpo_item* it) { return (i128)(((u128)(uint64_t)it->b_hi << 64) | it->b_lo); }
static i128 item_c(const mpo_item* it) { return (i128)(((u128)(uint64_t)it->c_hi << 64) | it->c_lo); }

static uint64_t mod128(i128 v, uint64_t n) {          /* Math.hpp:196-202 */
    i128 r = v % (i128)n;
    if (r < 0) r += (i128)n;
    return (uint64_t)r;
}
static uint64_t mod_neg(i128 v, uint64_t n) {         /* Math.hpp:204-207 */
    const uint64_t r = mod128(v, n);
    return r == 0 ? 0 : n - r;
}
static uint64_t isqrt_ceil_u64(uint64_t n) {          /* Math.hpp:146-174 */
    if (n == 0) return 0;
    uint64_t r = 0;
    for (int bit = 31; bit >= 0; --bit) {
        const uint64_t c = r | (1ULL << bit);
        if ((u128)c * c <= n) r = c;
    }
    return (u128)r * r < n ? r + 1 : r;
}
static uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) { const uint64_t t = a % b; a = b; b = t; }
    return a;
}

/* ---- multiplicative order, Math.hpp:253-310 ---- */
static uint64_t rho_brent(uint64_t n, uint64_t c) {
    /* Pollard-Brent with f(x) = x^2 + c mod n; returns a factor (maybe n). */
    uint64_t y = 2, x = 2, q = 1, g = 1, ys = 2;
    uint64_t r = 1;
    const uint64_t m = 64;
    while (g == 1) {
        x = y;
        for (uint64_t i = 0; i < r; ++i) y = (uint64_t)(((u128)y * y + c) % n);
        uint64_t k = 0;
        while (k < r && g == 1) {
            ys = y;
            const uint64_t lim = (m < r - k) ? m : r - k;
            for (uint64_t i = 0; i < lim; ++i) {
                y = (uint64_t)(((u128)y * y + c) % n);
                q = (uint64_t)(((u128)q * (x > y ? x - y : y - x)) % n);
            }
            g = gcd64(q, n);
            k += m;
        }
        r <<= 1;
    }
    if (g == n) {
        do {
            ys = (uint64_t)(((u128)ys * ys + c) % n);
            g = gcd64(x > ys ? x - ys : ys - x, n);
        } while (g == 1);
    }
    return g;
}

static void factor_rec(uint64_t n, uint64_t* f, int* nf) {
    if (n == 1) return;
    if (mpo_is_prime64(n)) { f[(*nf)++] = n; return; }
    if ((n & 1) == 0) { f[(*nf)++] = 2; factor_rec(n >> 1, f, nf); return; }
    uint64_t d = n;
    for (uint64_t c = 1; d == n || d == 1; ++c) d = rho_brent(n, c);
    factor_rec(d, f, nf);
    factor_rec(n / d, f, nf);
}

uint64_t mpo_mult_order(uint64_t b, uint64_t p) {
    uint64_t f[128];
    int nf = 0;
    uint64_t n = p - 1;
    for (uint64_t d = 2; d < 1000 && d * d <= n; ++d) {
        while (n % d == 0) { f[nf++] = d; n /= d; }
    }
    factor_rec(n, f, &nf);
    uint64_t order = p - 1;
    for (int i = 0; i < nf; ++i) {
        int dup = 0;
        for (int k = 0; k < i; ++k) dup |= (f[k] == f[i]);
        if (dup) continue;
        while (order % f[i] == 0 && mpo_powmod(b % p, order / f[i], p) == 1) order /= f[i];
    }
    return order;
}

/* ---- run_bsgs_reference, Math.hpp:488-542 (p < 1000, p even, p | b) ---- */
static int run_bsgs_reference(uint64_t p, const mpo_item* it, mpo_relation* out) {
    if (p < 2) return 0;
    const uint64_t b_mod = mod128(item_b(it), p);
    const uint64_t t = mod_neg(item_c(it), p);
    if (b_mod == 0) {
        if (t == 0) { out->p = p; out->M = (uint64_t)it->N0; out->q = 1; return 1; }
        return 0;
    }
    const i128 lim = ((i128)p > (i128)it->N1) ? (i128)it->N1 : (i128)p;
    if (lim <= 0) return 0;                       /* isqrt_ceil(<= 0) == 0 */
    const uint64_t m = isqrt_ceil_u64((uint64_t)lim);
    if (m == 0) return 0;
    /* The reference's baby map keeps the first i per value, and its giant
     * loop walks j upward: the result is the smallest n in [0, m*m) with
     * b^n == -c (mod p).  Here p < 1000 or p | b, so a direct walk is exact. */
    uint64_t v = 1 % p;
    for (uint64_t n = 0; n < m * m; ++n) {
        if (v == t) {
            out->p = p; out->M = n; out->q = mpo_mult_order(b_mod, p);
            return 1;
        }
        v = (uint64_t)(((u128)v * b_mod) % p);
    }
    return 0;
}

/* ---- exact BSGS core, Math.hpp:439-479 ----
 * Smallest j in [0, jcount) with B^j == target (Montgomery residues). */
static uint64_t bsgs_core(const mont* mt, uint64_t B, uint64_t target, uint64_t jcount, uint64_t* bsgs_mul) {
    uint64_t m = 1;
    while (m * m < jcount) ++m;   /* == ceil(sqrt(jcount)) as computed by Math.hpp:439-441 */
    baby_table* table = &tl_table;
    table_reset(table, m);
    const uint64_t before = tl_mul;
    uint64_t power = mt->one, cycle = 0;
    for (uint64_t i = 0; i < m; ++i) {
        if (i > 0 && power == mt->one) { cycle = i; break; }
        table_insert(table, power, (uint32_t)i);
        power = mont_mul(mt, power, B);
    }
    uint32_t idx = 0;
    uint64_t j = UINT64_MAX;
    if (cycle != 0) {
        if (table_find(table, target, &idx)) j = idx;
    } else {
        const uint64_t after_baby = tl_mul;
        const uint64_t step_inv = mont_pow(mt, power, mt->n - 2);
        const uint64_t pow_cost = tl_mul - after_baby;
        uint64_t giant = target;
        for (uint64_t g = 0; g * m < jcount; ++g) {
            if (table_find(table, giant, &idx)) { j = idx + g * m; break; }
            giant = mont_mul(mt, giant, step_inv);
        }
        if (bsgs_mul) *bsgs_mul -= pow_cost;   /* the inverse is set-up, not a step */
    }
    if (bsgs_mul) *bsgs_mul += tl_mul - before;
    return j < jcount ? j : UINT64_MAX;
}

uint64_t mpo_bsgs_smallest_j(uint64_t p, uint64_t B, uint64_t G0, uint64_t t, uint64_t jcount) {
    if (jcount == 0) return UINT64_MAX;
    mont mt;
    mont_init(&mt, p);
    /* G0 * B^j == t  <=>  B^j == t * G0^-1 */
    const uint64_t Bm = mont_to(&mt, B);
    const uint64_t tm = mont_mul(&mt, mont_to(&mt, t), mont_pow(&mt, mont_to(&mt, G0), p - 2));
    return bsgs_core(&mt, Bm, tm, jcount, NULL);
}

/* ---- run_bsgs, Math.hpp:377-486 ---- */
static int run_bsgs_counted(uint64_t p, const mpo_item* it, mpo_relation* out,
                            uint64_t* prep_mul, uint64_t* bsgs_mul, uint64_t* reached) {
    if (p < 1000 || p >= (1ULL << 62) || (p & 1) == 0) return run_bsgs_reference(p, it, out);
    const uint64_t b_mod = mod128(item_b(it), p);
    const uint64_t t = mod_neg(item_c(it), p);
    if (b_mod == 0) return run_bsgs_reference(p, it, out);
    if (t == 0) return 0;

    const uint64_t N0 = it->N0 < 0 ? 0 : (uint64_t)it->N0;
    const uint64_t N1 = (uint64_t)it->N1;
    const uint64_t cm = it->mod == 0 ? 1 : it->mod;
    const uint64_t n_start = N0 + ((it->res % cm) + cm - (N0 % cm)) % cm;
    if (n_start >= N1) return 0;
    uint64_t kcount = (N1 - n_start + cm - 1) / cm;
    if (kcount > p) kcount = p;

    const uint64_t mul0 = tl_mul;
    mont mt;
    mont_init(&mt, p);
    const uint64_t b_m = mont_to(&mt, b_mod);
    uint64_t B = mont_pow(&mt, b_m, cm);
    uint64_t target = mont_to(&mt, t);
    if (n_start != 0) target = mont_mul(&mt, target, mont_pow(&mt, mont_pow(&mt, b_m, n_start), p - 2));

    uint64_t stride = 1, parity = 0;
    const uint64_t g = gcd64(cm, p - 1);
    int pass = 1;
    if (g >= 2) {
        if (mont_pow(&mt, target, (p - 1) / g) != mt.one) pass = 0;
    } else {
        const int lb = mont_legendre(&mt, B);
        const int lt = mont_legendre(&mt, target);
        if (lb == 1) {
            if (lt == -1) pass = 0;
        } else {
            stride = 2;
            if (lt == -1) {
                parity = 1;
                target = mont_mul(&mt, target, mont_pow(&mt, B, p - 2));
            }
            B = mont_mul(&mt, B, B);
        }
    }
    if (prep_mul) *prep_mul += tl_mul - mul0;
    if (!pass || kcount <= parity) return 0;
    const uint64_t jcount = (kcount - parity + stride - 1) / stride;
    if (reached) ++*reached;

    const uint64_t mul1 = tl_mul;
    uint64_t bm = 0;
    const uint64_t j = bsgs_core(&mt, B, target, jcount, &bm);
    if (prep_mul) *prep_mul += (tl_mul - mul1) - bm;   /* the B^-m inverse */
    if (bsgs_mul) *bsgs_mul += bm;
    if (j == UINT64_MAX) return 0;

    const uint64_t k = j * stride + parity;
    out->p = p;
    out->M = n_start + k * cm;
    out->q = mpo_mult_order(b_mod, p);
    return 1;
}

int mpo_run_bsgs(uint64_t p, const mpo_item* it, mpo_relation* out) {
    return run_bsgs_counted(p, it, out, NULL, NULL, NULL);
}

/* ---- sieve, Sieve.hpp:13-185 ---- */
static pthread_mutex_t sp_lock = PTHREAD_MUTEX_INITIALIZER;
static uint32_t* sp_list;         /* primes <= sp_limit, ascending */
static size_t sp_count;
static uint64_t sp_limit;

/* Sieve.hpp:13-39: primes up to limit (cached, grows on demand). */
static void small_primes(uint64_t limit, const uint32_t** list, size_t* count) {
    pthread_mutex_lock(&sp_lock);
    if (sp_list == NULL || sp_limit < limit) {
        uint64_t lim = limit < 65536 ? 65536 : limit;
        uint8_t* comp = (uint8_t*)calloc(lim + 1, 1);
        size_t n = 0;
        for (uint64_t i = 2; i <= lim; ++i) {
            if (comp[i]) continue;
            ++n;
            for (uint64_t j = i * i; j <= lim; j += i) comp[j] = 1;
        }
        uint32_t* out = (uint32_t*)malloc(n * sizeof(uint32_t));
        n = 0;
        for (uint64_t i = 2; i <= lim; ++i) if (!comp[i]) out[n++] = (uint32_t)i;
        free(comp);
        free(sp_list);
        sp_list = out; sp_count = n; sp_limit = lim;
    }
    *list = sp_list;
    *count = sp_count;
    pthread_mutex_unlock(&sp_lock);
}

/* Marks odd composites of [lo, hi) in a byte per odd with the given primes,
 * each from max(q^2, first odd multiple >= lo) (Sieve.hpp:49-107). */
typedef void (*emit_fn)(uint64_t v, void* ctx);

static void odd_sieve(uint64_t lo, uint64_t hi, uint64_t qmax, emit_fn emit, void* ctx) {
    /* lo odd, lo >= 3 */
    const uint32_t* sp;
    size_t nsp;
    small_primes(qmax, &sp, &nsp);
    const uint64_t seg = 1ULL << 18;
    uint8_t* z = (uint8_t*)malloc(seg);
    for (uint64_t s0 = lo; s0 < hi; s0 += 2 * seg) {
        const uint64_t s1 = (hi - s0 + 1) / 2 < seg ? hi : s0 + 2 * seg;
        const uint64_t len = (s1 - s0 + 1) / 2;
        memset(z, 0, len);
        for (size_t k = 1; k < nsp; ++k) {           /* skip 2 */
            const uint64_t q = sp[k];
            if (q > qmax) break;
            if (q * q >= s1) break;
            uint64_t start = ((s0 + q - 1) / q) * q;
            if (start < q * q) start = q * q;
            if ((start & 1) == 0) start += q;
            for (uint64_t v = (start - s0) / 2; v < len; v += q) z[v] = 1;
        }
        for (uint64_t i = 0; i < len; ++i) if (!z[i]) emit(s0 + 2 * i, ctx);
    }
    free(z);
}

typedef struct vec_ctx { uint64_t* out; size_t cap; size_t n; } vec_ctx;
static void emit_vec(uint64_t v, void* c) {
    vec_ctx* x = (vec_ctx*)c;
    if (x->n < x->cap) x->out[x->n] = v;
    ++x->n;
}

/* Exact primes of [lo, hi): the odd sieve by the primes up to
 * min(sqrt(hi), 65521), then is_prime64 on the survivors when sqrt(hi)
 * exceeds 65521 (Sieve.hpp:110-145 gives the same list with a full table of
 * small primes; Worker.hpp:222-227 filters GPU survivors the same way). */
typedef struct prime_filter_ctx { emit_fn emit; void* ctx; } prime_filter_ctx;
static void emit_if_prime(uint64_t v, void* c) {
    prime_filter_ctx* f = (prime_filter_ctx*)c;
    if (mpo_is_prime64(v)) f->emit(v, f->ctx);
}
static void odd_primes(uint64_t lo, uint64_t hi, emit_fn emit, void* ctx) {
    uint64_t l = lo < 3 ? 3 : (lo | 1);
    if (l >= hi) return;
    const uint64_t r = isqrt_ceil_u64(hi);
    if (r <= 65521) {
        odd_sieve(l, hi, r, emit, ctx);
    } else {
        prime_filter_ctx f = {emit, ctx};
        odd_sieve(l, hi, 65521, emit_if_prime, &f);
    }
}

size_t mpo_sieve(uint64_t lo, uint64_t hi, uint64_t* out, size_t cap) {
    vec_ctx x = {out, cap, 0};
    if (lo >= hi) return 0;
    if (lo <= 2 && hi > 2) emit_vec(2, &x);
    odd_primes(lo, hi, emit_vec, &x);
    return x.n;
}

size_t mpo_sieve_survivors(uint64_t lo, uint64_t hi, uint64_t* out, size_t cap) {
    vec_ctx x = {out, cap, 0};
    uint64_t l = lo < 3 ? 3 : (lo | 1);
    if (l < hi) odd_sieve(l, hi, 65521, emit_vec, &x);
    return x.n;
}

/* ---- Worker.hpp:195-303, CPU branch ---- */
typedef struct chunk_ctx {
    const mpo_item* item;
    mpo_relation* out;
    size_t cap, n;
    mpo_counts* counts;
    int survivors_mode;       /* 1: emit() receives sieve survivors (counted run) */
} chunk_ctx;

static void emit_prime(uint64_t p, void* c) {
    chunk_ctx* x = (chunk_ctx*)c;
    mpo_relation r;
    int is_prime = 1;
    if (x->survivors_mode) {
        const uint64_t m0 = tl_mul;
        is_prime = mpo_is_prime64(p);
        if (x->counts) x->counts->mr_mmul += tl_mul - m0;
    }
    if (!is_prime) return;
    if (x->counts) ++x->counts->primes;
    int hit;
    if (x->counts) hit = run_bsgs_counted(p, x->item, &r, &x->counts->prep_mmul, &x->counts->bsgs_mmul,
                                          &x->counts->bsgs_primes);
    else hit = run_bsgs_counted(p, x->item, &r, NULL, NULL, NULL);
    if (hit) {
        if (x->n < x->cap) x->out[x->n] = r;
        ++x->n;
    }
}

static size_t chunk_relations(uint64_t lo, uint64_t hi, const mpo_item* item, mpo_relation* out,
                              size_t cap, mpo_counts* counts) {
    chunk_ctx x = {item, out, cap, 0, counts, 0};
    if (lo >= hi) return 0;
    if (lo <= 2 && hi > 2) emit_prime(2, &x);
    uint64_t l = lo < 3 ? 3 : (lo | 1);
    if (l < hi) {
        if (counts) {
            counts->odds += (hi - l + 1) / 2;
            /* survivors of the sieve by 3..65521 go through is_prime64 as on the
             * GPU path (Worker.hpp:222-227); exact primes result either way */
            x.survivors_mode = 1;
            const uint64_t qmax = isqrt_ceil_u64(hi) < 65521 ? isqrt_ceil_u64(hi) : 65521;
            odd_sieve(l, hi, qmax, emit_prime, &x);
        } else {
            odd_primes(l, hi, emit_prime, &x);
        }
    }
    if (counts) counts->relations += x.n;
    return x.n;
}

size_t mpo_chunk_relations(uint64_t lo, uint64_t hi, const mpo_item* item, mpo_relation* out, size_t cap) {
    return chunk_relations(lo, hi, item, out, cap, NULL);
}

size_t mpo_chunk_relations_counted(uint64_t lo, uint64_t hi, const mpo_item* item, mpo_relation* out,
                                   size_t cap, mpo_counts* counts) {
    return chunk_relations(lo, hi, item, out, cap, counts);
}

/* ---- threaded driver, Worker.hpp:305-367 ---- */
typedef struct pool {
    uint64_t lo, hi, chunk;
    const mpo_item* item;
    pthread_mutex_t lock;
    uint64_t next;
    mpo_relation* rel;
    size_t n, cap;
} pool;

static void* pool_worker(void* arg) {
    pool* P = (pool*)arg;
    size_t bcap = 1024;
    mpo_relation* buf = (mpo_relation*)malloc(bcap * sizeof(mpo_relation));
    for (;;) {
        pthread_mutex_lock(&P->lock);
        const uint64_t lo = P->next;
        if (lo >= P->hi) { pthread_mutex_unlock(&P->lock); break; }
        const uint64_t hi = (P->hi - lo > P->chunk) ? lo + P->chunk : P->hi;
        P->next = hi;
        pthread_mutex_unlock(&P->lock);
        size_t k = chunk_relations(lo, hi, P->item, buf, bcap, NULL);
        if (k > bcap) {
            bcap = k;
            buf = (mpo_relation*)realloc(buf, bcap * sizeof(mpo_relation));
            k = chunk_relations(lo, hi, P->item, buf, bcap, NULL);
        }
        pthread_mutex_lock(&P->lock);
        for (size_t i = 0; i < k; ++i) {
            if (P->n < P->cap) P->rel[P->n] = buf[i];
            ++P->n;
        }
        pthread_mutex_unlock(&P->lock);
    }
    free(buf);
    return NULL;
}

static int rel_cmp(const void* a, const void* b) {
    const mpo_relation* x = (const mpo_relation*)a;
    const mpo_relation* y = (const mpo_relation*)b;
    return x->p < y->p ? -1 : x->p > y->p ? 1 : 0;
}

size_t mpo_relations_threaded(uint64_t lo, uint64_t hi, const mpo_item* item, mpo_relation* out,
                              size_t cap, int threads, uint64_t chunk) {
    if (threads < 1) threads = 1;
    if (chunk == 0) chunk = 1ULL << 24;
    pool P;
    P.lo = lo; P.hi = hi; P.chunk = chunk; P.item = item; P.next = lo;
    P.rel = out; P.n = 0; P.cap = cap;
    pthread_mutex_init(&P.lock, NULL);
    const uint32_t* sp; size_t nsp;
    small_primes(65536, &sp, &nsp);   /* build the cache once, before the threads */
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, pool_worker, &P);
    for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    free(th);
    pthread_mutex_destroy(&P.lock);
    const size_t kept = P.n < cap ? P.n : cap;
    qsort(out, kept, sizeof(mpo_relation), rel_cmp);
    return P.n;
}
