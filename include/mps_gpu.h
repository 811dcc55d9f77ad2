/*
 * mps_gpu.h -- C-ABI of the B200 (sm_100a) Mass Prime Siever worker.
 *
 * Drop-in boundary for the GPU worker of Mass Prime Siever 14.0.  The
 * reference binds its GPU through the C++ class GpuSiever
 * ("Mass Prime Siever/Gpu.hpp":1040-1074) with two calls, sieve_filter and
 * filter, made by process_chunk ("Mass Prime Siever/Worker.hpp":195-303).
 * This header exposes the same two contracts as plain C functions, plus the
 * exact relation path that moves run_bsgs ("Mass Prime Siever/Math.hpp":
 * 377-486) onto the device, and a batched entry point for many items.
 *
 * Conventions: every function returns MPS_OK (0) or a negative MPS_E_* code;
 * mps_last_error(ctx) gives the reason as text.  Buffers are caller-owned
 * host memory; the library owns its device memory, allocated on demand and
 * released by mps_close.  A context is used by one host thread at a time
 * (the reference serialises its feeder threads with a mutex, Gpu.hpp:1059).
 */
#ifndef MPS_GPU_H
#define MPS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPS_ABI_VERSION 1

enum {
    MPS_OK = 0,
    MPS_E_ARG = -1,       /* malformed arguments (NULL, P0 >= P1, res >= mod, ...)        */
    MPS_E_RANGE = -2,     /* outside the GPU path: P1 > 2^62, lo <= 3 (compat), N1-N0 > 1e7 */
    MPS_E_CAPACITY = -3,  /* the caller's output buffer is too small (*n_out = needed)     */
    MPS_E_TIMEOUT = -4,   /* a bounded device wait expired                                */
    MPS_E_CUDA = -5,      /* a CUDA call failed                                           */
    MPS_E_NODEV = -6,     /* no usable CUDA device                                        */
    MPS_E_STATE = -7      /* the context is closed or was poisoned by an earlier error    */
};

typedef struct mps_ctx mps_ctx;

/* One Factor=b,c,P0,P1,N0,N1[,mod,res] line (Config.hpp:124-200, Types.hpp:14-26).
 * b and c are signed 128-bit integers (two's complement, high word signed). */
typedef struct mps_item {
    int64_t  b_hi;
    uint64_t b_lo;
    int64_t  c_hi;
    uint64_t c_lo;
    uint64_t P0, P1;      /* primes P0 <= p < P1, P1 <= 2^62                 */
    int64_t  N0, N1;      /* exponents N0 <= n < N1, N1 - N0 <= 10^7         */
    uint64_t mod, res;    /* n == res (mod mod); mod 0 is taken as 1         */
} mps_item;

/* A relations.p line "p, M, q": p | b^n + c for n == M (mod q)
 * (Math.hpp:360-364, Worker.hpp:294-297). */
typedef struct mps_relation {
    uint64_t p, M, q;
} mps_relation;

/* Tuning; mps_tuning_default fills the defaults (zero fields take them too, except table_kind,
 * whose zero is a kind of its own).  Every setting gives the same relations. */
typedef struct mps_tuning {
    uint32_t struct_size;       /* sizeof(mps_tuning)                                          */
    uint32_t table_bits;        /* baby-step table of 2^bits slots per prime (0: per item)     */
    uint64_t chunk_odds;        /* odd integers per device chunk (0: 2^26)                      */
    uint32_t max_baby;          /* cap on the baby-step count (0: what the table holds)        */
    uint32_t bsgs_warps;        /* warps per BSGS block (0: 4)                                 */
    uint32_t class_modulus;     /* Q of the power-residue split g = gcd(Q, p-1), even, <= 2^28
                                   (0: lcm(mod, 232792560), else lcm(mod, 720720), else
                                    lcm(mod, 5040), the first within 2^28, else 5040;
                                    1: lcm(mod, 2), the reference's plain-method filter)       */
    uint32_t full_mr;           /* 1: 12-base Miller-Rabin on every filter survivor (eager)    */
    uint32_t plain;             /* 1: plain per-chunk path (host sync between stages)          */
    uint32_t chains;            /* BSGS chains per lane, 1, 2 or 4 (0: 2)                      */
    uint32_t graphs_off;        /* 1: launch waves directly instead of replaying CUDA graphs   */
    uint32_t table_kind;        /* BSGS table: 0 = four 16-bit fingerprints per 64-bit word,
                                   inserted by compare-and-swap, 1 = one 32-bit key per slot,
                                   2 = one 16-bit fingerprint per slot, read with one 16-bit
                                   load per probe, 3 = the words of 0 with a count byte per
                                   word, a half claimed by one atomic add (the default)     */
    uint32_t load_shift;        /* table kind 2: a prime's table has at least 2^load_shift
                                   slots per baby step (0: 2)                                   */
    uint32_t lanes;             /* table kind 2: lanes per prime, 32, 16 or 8 (0: 32); groups of
                                   16 or 8 solve 2 or 4 primes per warp, for p < 2^49          */
    uint32_t table_fill;        /* table kinds 0 and 3: at most table_fill/256 keys per 64-bit
                                   word on average, 1..256 (0: 160)                            */
    uint32_t baby_scale;        /* baby steps m = ceil(sqrt(j range) * baby_scale / 256) before
                                   the table's cap, 1..1024 (0: 160; 256 is the square root)   */
} mps_tuning;

/* Counters of the last call (all chunks of it). */
typedef struct mps_stats {
    uint64_t odds;              /* odd integers sieved                          */
    uint64_t survivors;         /* survivors of the sieve by the primes <= 65521 */
    uint64_t entries;           /* primes that reached the BSGS                 */
    uint64_t relations;         /* relations returned                           */
    uint64_t chunks;            /* device chunks run                            */
    double   device_ms;         /* device time of the call (CUDA events)        */
    double   bsgs_ms;           /* device time of the BSGS kernel               */
    uint64_t bsgs_launches;
    uint64_t kernel_launches;   /* kernels of this library launched             */
    uint64_t bsgs_steps;        /* baby + giant steps (Montgomery multiplies) done by the BSGS */
    double   sieve_ms;          /* device time of the sieve kernel (CUDA events)  */
    double   prep_ms;           /* device time of the prep kernel                 */
    double   order_ms;          /* device time of the order kernel                */
    uint64_t bsgs_baby_steps;   /* the baby steps among bsgs_steps                */
} mps_stats;

/* ---- context (replaces CudaSiever::init, Cuda.hpp:198-257) ---- */
int mps_tuning_default(mps_tuning* t);
int mps_open(int device, const mps_tuning* tuning, mps_ctx** out);
int mps_close(mps_ctx* ctx);
const char* mps_last_error(const mps_ctx* ctx);
int mps_get_stats(const mps_ctx* ctx, mps_stats* out);
int mps_abi_version(void);

/* ---- the exact path (new): run_bsgs on every prime of [lo, hi), on the device ----
 * Relations of the primes lo <= p < hi, sorted by p.  0 <= lo < hi <= 2^62; the
 * item's own P0/P1 are not consulted.  If cap is too small, returns
 * MPS_E_CAPACITY with *n_out = the number needed.  Replaces the CPU loop of
 * process_chunk (Worker.hpp:243-280) for one chunk. */
int mps_chunk_relations(mps_ctx* ctx, uint64_t lo, uint64_t hi, const mps_item* item,
                        mps_relation* out, size_t cap, size_t* n_out);

/* All relations of one item, p over [P0, P1) (run_worker_pool, Worker.hpp:305-367). */
int mps_item_relations(mps_ctx* ctx, const mps_item* item, mps_relation* out, size_t cap, size_t* n_out);

/* ---- compat: GpuSiever::sieve_filter (Gpu.hpp:1064-1067, Cuda.hpp:329-415) ----
 * Appends to out the numbers of [lo, hi) that may divide an in-class
 * candidate: here exactly the primes with a relation, ascending.  Declines
 * with MPS_E_RANGE unless hi < 2^62 and lo > 3 (Worker.hpp:209). */
int mps_sieve_filter(mps_ctx* ctx, uint64_t lo, uint64_t hi, const mps_item* item,
                     uint64_t* out, size_t cap, size_t* n_out);

/* ---- compat: GpuSiever::filter (Gpu.hpp:1060-1063, Cuda.hpp:264-326) ----
 * flags[i] = 1 when primes[i] may divide an in-class candidate (here: exactly
 * when it has a relation), else 0.  primes[] are host-sieved primes. */
int mps_filter(mps_ctx* ctx, const uint64_t* primes, size_t n, const mps_item* item, uint8_t* flags);

/* ---- batched: many items through one persistent work-stealing launch per chunk ----
 * Relations of every item over its [P0, P1); out_item[k] is the item index of
 * out[k]; sorted by (item, p). */
int mps_batch_relations(mps_ctx* ctx, const mps_item* items, size_t n_items, mps_relation* out,
                        uint32_t* out_item, size_t cap, size_t* n_out);

/* The relations of the last mps_chunk_relations / mps_item_relations /
 * mps_batch_relations call again, without recomputing them: after such a call
 * returned MPS_E_CAPACITY (with *n_out = the count), pass a buffer of that
 * size here.  out_item may be NULL. */
int mps_take_relations(mps_ctx* ctx, mps_relation* out, uint32_t* out_item, size_t cap, size_t* n_out);

/* ---- serving: continuous batching of Factor= items (no counterpart in the reference) ----
 * A server owns a device context, a worker thread and a device pool of
 * min(mem_budget_bytes, 90% of the free device memory), allocated by
 * mps_serve_open.  Every admitted item holds a reservation in that pool: a
 * device buffer for its relations, sized at twice its expected relation
 * count plus 256, which the commit kernel fills wave by wave (the item's
 * device-resident result; a result that outgrows it comes from the host copy
 * of the wave results instead).  Submitted items wait, in arrival order,
 * until fewer than max_active are in flight and their reservation fits in
 * the pool; an item larger than the whole pool fails with MPS_E_CAPACITY.
 * Every wave takes one piece of piece_odds odd numbers from each in-flight
 * item in turn, so items that arrive while others run join the next wave;
 * the sieve segments, BSGS entries and baby-step tables of a wave live in
 * the server's two fixed wave buffers.  Per-item progress is kept in a
 * device table (mps_serve_checkpoint).  Results equal mps_item_relations on
 * the same item. */
typedef struct mps_server mps_server;
typedef struct mps_serve_config {
    uint32_t struct_size;       /* sizeof(mps_serve_config)                  */
    uint32_t max_active;        /* items in flight at once (0: 256)           */
    uint64_t mem_budget_bytes;  /* device memory for in-flight items (0: 4 GiB) */
    uint64_t piece_odds;        /* odd numbers per item piece (0: 2^22)       */
    uint32_t reserved[8];
} mps_serve_config;
typedef struct mps_serve_status {
    uint64_t ticket;
    int32_t  state;             /* 0 queued, 1 running, 2 done, 3 failed      */
    int32_t  error;
    uint64_t p_done;
    uint64_t relations;
    double   latency_ms;        /* submit -> done                             */
    double   queue_ms;          /* submit -> admitted                         */
    uint64_t reserved_bytes;    /* the item's reservation in the device pool  */
    int32_t  relations_on_device; /* 1: the result was read from its device buffer */
    int32_t  pad;
} mps_serve_status;
int mps_serve_config_default(mps_serve_config* cfg);
int mps_serve_open(int device, const mps_tuning* tuning, const mps_serve_config* cfg, mps_server** out);
int mps_serve_submit(mps_server* sv, const mps_item* item, uint64_t* ticket);
/* MPS_OK when done, MPS_E_TIMEOUT if still running after timeout_s. */
int mps_serve_wait(mps_server* sv, uint64_t ticket, double timeout_s, mps_serve_status* status);
int mps_serve_result(mps_server* sv, uint64_t ticket, mps_relation* out, size_t cap, size_t* n_out);
int mps_serve_release(mps_server* sv, uint64_t ticket);
/* The reservation pool: its size, the bytes reserved by admitted items, and
 * the items in flight and waiting. */
int mps_serve_pool(mps_server* sv, uint64_t* pool_bytes, uint64_t* reserved_bytes, uint32_t* active,
                   uint32_t* queued);
/* Device-resident progress of an item: every p below *p_done sieved, *n_rel relations. */
int mps_serve_checkpoint(mps_server* sv, uint64_t ticket, uint64_t* p_done, uint64_t* n_rel);
int mps_serve_close(mps_server* sv);

/* ---- autotuner (no counterpart in the reference, which sizes its baby-step table per
 * item, Cuda.hpp:342-348, and picks m and Gc per prime, Gpu.hpp:553-573) ----
 * For every item class among items -- the bit length of K (the item's count of
 * in-class exponents), the class modulus, the decimal digits of P0 -- times
 * each candidate BSGS configuration (table kind, table load, lanes per prime,
 * chains per lane, warps per block) by the BSGS kernel's CUDA events on a calibration slice of
 * the item (its first 2^25 integers); with the fastest, the table fill and the
 * baby/giant balance (baby_scale) the same way; then the sieve's segment size
 * (1024, 2048 or 4096 words) by the sieve kernel's events;
 * checks that every candidate gives the same relations, and keeps the
 * fastest configuration for the class.  Later calls on items of a tuned class
 * use it (per item; a batched wave uses the configuration of its item with
 * the largest K).  One report per class tuned; MPS_E_CAPACITY if cap is too
 * small (*n_out = the number of classes).  The tuning changes speed only:
 * relations are identical under every configuration. */
typedef struct mps_tune_report {
    uint32_t k_bits;              /* class: bit length of K                              */
    uint32_t mod;                 /* class: class modulus (capped at 4095)               */
    uint32_t p_digits;            /* class: decimal digits of P0, minus one              */
    uint32_t candidates;          /* configurations timed                                */
    uint32_t table_kind, load_shift, chains, warps;   /* the BSGS configuration chosen   */
    uint32_t seg_words;           /* the sieve segment chosen (words of 32 odd numbers)  */
    uint32_t lanes;               /* lanes per prime chosen (32, or groups of 16 or 8)   */
    uint32_t table_fill;          /* table load chosen (keys per word x 256)             */
    uint32_t baby_scale;          /* baby-step scale chosen (x 256 of the square root)   */
    double   best_ns_per_prime;   /* BSGS time per prime reaching the BSGS, chosen       */
    double   default_ns_per_prime;/* the same under the context's tuning fields          */
    double   sieve_best_ms;       /* sieve time of the calibration slice, chosen segment */
    double   sieve_default_ms;    /* the same with the default segment (2048 words)      */
    uint64_t calib_bsgs_primes;   /* primes of the calibration slice reaching the BSGS   */
} mps_tune_report;
int mps_autotune(mps_ctx* ctx, const mps_item* items, size_t n_items, mps_tune_report* out, size_t cap,
                 size_t* n_out);
/* The tuned classes as text ("mps-tune 4" then one line per class); mps_open
 * loads the file named by the environment variable MPS_TUNE_CACHE, if set. */
int mps_tune_save(const mps_ctx* ctx, const char* path);
int mps_tune_load(mps_ctx* ctx, const char* path);
int mps_tune_clear(mps_ctx* ctx);

/* Number of primes in [lo, hi) counted on the device (the unit of the
 * sieved-primes/s metric; not part of the relation path). */
int mps_count_primes(mps_ctx* ctx, uint64_t lo, uint64_t hi, uint64_t* count);

/* Arithmetic ceilings measured on this device, from independent chains:
 * exact FP64-pipe modular multiplies per second (the step of every BSGS
 * with p < 2^49), 64-bit integer Montgomery multiplies per second (p >=
 * 2^49), and 32-bit integer multiply-adds per second (the integer pipe). */
int mps_measure_peaks(mps_ctx* ctx, double* fmul_per_s, double* mmul_per_s, double* imad_per_s);

/* Shared-memory ceiling of the segment sieve, measured on this device:
 * conflict-free 32-bit shared-memory atomicOr operations per second. */
int mps_measure_smem_peak(mps_ctx* ctx, double* atomic_or_per_s);

/* ---- relations of one small range without allocating (no counterpart in the reference) ----
 * For callers that cannot allocate device memory where they sieve: their
 * device memory belongs to another framework's pool allocator, or cudaMalloc
 * / cudaFree (which synchronise the device) are not allowed in their loop.
 * Same relations as mps_chunk_relations with the default tuning (its BSGS
 * runs table kind 0, which needs no count bytes, with the default fill and
 * baby-step scale), on the calling thread's current device and its
 * per-thread default stream
 * (cudaStreamPerThread), with no context.  All scratch is one static device
 * array of 8 MiB that every GPU loading this library holds until exit; its
 * address is looked up on the first call on each device (make that first
 * call before any stream capture).  Calls on one device share its array, so
 * two calls that overlap on the same GPU race and must not be made; calls on
 * different devices may overlap.  hi - lo must not exceed 2^19 (MPS_E_RANGE
 * otherwise); hi <= 2^62. */
int mps_chunk_relations_noalloc(uint64_t lo, uint64_t hi, const mps_item* item,
                                mps_relation* out, size_t cap, size_t* n_out);

/* ---- kernel-level hooks for parity tests ---- */
/* Survivors of the odd sieve of [lo, hi) by the odd primes <= min(65521, sqrt(hi)), ascending. */
int mps_test_survivors(mps_ctx* ctx, uint64_t lo, uint64_t hi, uint64_t* out, size_t cap, size_t* n_out);
/* out[i] = is_prime64(n[i]) (Math.hpp:209-251), n[i] < 2^62. */
int mps_test_is_prime(mps_ctx* ctx, const uint64_t* n, size_t count, uint8_t* out);
/* cases[5k..5k+4] = p, B, G0, t, jcount: smallest j < jcount with G0*B^j == t (mod p),
 * or UINT64_MAX; B, G0, t in [1, p). */
int mps_test_bsgs(mps_ctx* ctx, const uint64_t* cases, size_t count, uint32_t table_bits, uint64_t* j_out);
/* bp[2k], bp[2k+1] = b, p (p prime, p does not divide b): q_out[k] = ord_p(b) (Math.hpp:294-310). */
int mps_test_order(mps_ctx* ctx, const uint64_t* bp, size_t count, uint64_t* q_out);

#ifdef __cplusplus
}
#endif
#endif
