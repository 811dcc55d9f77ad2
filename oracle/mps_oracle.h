/*
 * mps_oracle.h -- CPU restatement of the Mass Prime Siever 14.0 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the sm_100a
 * kernels: tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * may call it, nothing in the product links it.  Every function names the
 * reference source it restates ("Mass Prime Siever/<file>:<line>").
 *
 * Parity pin: the restatement is checked against relations produced by the
 * reference's own Math.hpp/Sieve.hpp (compiled by oracle/Makefile into
 * oracle/_ref/) and committed as golden fixtures under tests/golden/.
 */
#ifndef MPS_ORACLE_H
#define MPS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One Factor= work item.  b and c are signed 128-bit integers split into a
 * two's-complement high word and a low word (the reference keeps them as
 * boost int128_t, Types.hpp:14-26).  mod == 0 is treated as 1. */
typedef struct mpo_item {
    int64_t  b_hi;
    uint64_t b_lo;
    int64_t  c_hi;
    uint64_t c_lo;
    uint64_t P0, P1;
    int64_t  N0, N1;
    uint64_t mod, res;
} mpo_item;

/* relations.p line "p, M, q" (Math.hpp:360-364, Worker.hpp:294-297). */
typedef struct mpo_relation {
    uint64_t p, M, q;
} mpo_relation;

/* Work counters of the reference algorithm, for the roofline's algorithmic
 * operation count.  Counted per call of mpo_chunk_relations_counted. */
typedef struct mpo_counts {
    uint64_t odds;          /* odd integers in the chunk                         */
    uint64_t primes;        /* primes in the chunk                               */
    uint64_t mr_mmul;       /* modular multiplies of is_prime64 on every prime   */
    uint64_t prep_mmul;     /* run_bsgs set-up + residue filter multiplies       */
    uint64_t bsgs_mmul;     /* baby + giant step multiplies                      */
    uint64_t bsgs_primes;   /* primes that reached the baby-step table           */
    uint64_t relations;
} mpo_counts;

/* Math.hpp:209-251: deterministic 12-base Miller-Rabin. */
int mpo_is_prime64(uint64_t n);

/* Binary Jacobi symbol (a/n), n odd (Gpu.hpp:213-226). */
int mpo_jacobi(uint64_t a, uint64_t n);

/* Montgomery constants for odd n < 2^63 (Math.hpp:35-45). */
void mpo_mont_consts(uint64_t n, uint64_t* ninv, uint64_t* one, uint64_t* r2);
/* Montgomery product a*b*2^-64 mod n (Math.hpp:47-61). */
uint64_t mpo_mont_mul(uint64_t a, uint64_t b, uint64_t n, uint64_t ninv);
/* a^e mod n, plain residues (Math.hpp:126-140). */
uint64_t mpo_powmod(uint64_t a, uint64_t e, uint64_t n);

/* All primes in [lo, hi), ascending (Sieve.hpp:110-185).  Writes at most
 * cap of them; returns the number of primes in the range. */
size_t mpo_sieve(uint64_t lo, uint64_t hi, uint64_t* out, size_t cap);

/* Survivors of the odd sieve by the odd primes 3..65521: every odd v in
 * [lo, hi), v >= 3, with no odd prime factor q <= 65521 other than v
 * itself (Gpu.hpp:385-455 semantics).  Returns the count. */
size_t mpo_sieve_survivors(uint64_t lo, uint64_t hi, uint64_t* out, size_t cap);

/* Math.hpp:294-310: order of b modulo the prime p. */
uint64_t mpo_mult_order(uint64_t b, uint64_t p);

/* Math.hpp:377-486 (and :488-542 for the small/degenerate primes): the
 * relation of one prime, 1 if there is one. */
int mpo_run_bsgs(uint64_t p, const mpo_item* item, mpo_relation* out);

/* Smallest j in [0, jcount) with G0 * B^j == t (mod p), or UINT64_MAX.
 * Plain residues; the exact BSGS of Math.hpp:439-479 on given inputs. */
uint64_t mpo_bsgs_smallest_j(uint64_t p, uint64_t B, uint64_t G0, uint64_t t, uint64_t jcount);

/* Worker.hpp:195-303 (CPU branch): every relation of the primes in
 * [lo, hi), in ascending p.  Returns the number of relations; writes at
 * most cap.  Thread-safe. */
size_t mpo_chunk_relations(uint64_t lo, uint64_t hi, const mpo_item* item,
                           mpo_relation* out, size_t cap);
size_t mpo_chunk_relations_counted(uint64_t lo, uint64_t hi, const mpo_item* item,
                                   mpo_relation* out, size_t cap, mpo_counts* counts);

/* Same over [lo, hi) with `threads` POSIX threads over chunks of `chunk`
 * integers (Worker.hpp:305-367); relations sorted by p. */
size_t mpo_relations_threaded(uint64_t lo, uint64_t hi, const mpo_item* item,
                              mpo_relation* out, size_t cap, int threads, uint64_t chunk);

#ifdef __cplusplus
}
#endif
#endif
