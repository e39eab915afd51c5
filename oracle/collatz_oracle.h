/*
 * collatz_oracle.h -- CPU oracle for the collatz_b200 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline / reference legs of
 * bench.py load it.  The product library (collatz_b200/) never links,
 * loads or calls it, and nothing in the product falls back to it.
 *
 * Three modes:
 *   cases  -- a plain-C restatement of the reference's Algorithm 1
 *             (collatz_cudav7.cu: THREEPOWERS cu:104-105, magic numbers
 *             cu:122-128, precompute cu:423-495, search1 cu:497-563,
 *             compute_kernel cu:185-411, search2/search3 cu:654-715).
 *             Pinned against the reference compiled here through a CPU
 *             shim (oracle/build_ref.sh) -> tests/golden/.
 *   range  -- every seed n in [offset, offset+size) that survives the
 *             k-step descent sieve and the mod-9 sieve is iterated until
 *             it falls below its start (new entry mode; outputs pinned
 *             only by this oracle: a single-step and a run-length
 *             formulation are checked against each other).
 *   traj   -- per-seed stopping time and maximum excursion for arbitrary
 *             seeds up to 256 bits (values up to 512 bits).
 *
 * Definitions used throughout (T is the reference's map, rs:13):
 *   T(n) = (3n+1)/2 for odd n, n/2 for even n.
 *   sigma(n) = least k >= 1 with T^k(n) < n (stopping time).
 *   E(n)     = max_{0<=k<=sigma(n)} T^k(n) (maximum excursion).
 *   Cases mode only sees T^k(n) for k >= N-A (Step 1 does not carry
 *   per-seed history), so there E is the max over N-A <= k <= sigma and
 *   sigma counts from n.  Ties in either maximum go to the smaller seed.
 */
#ifndef COLLATZ_ORACLE_H
#define COLLATZ_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned __int128 orc_u128;

#define ORC_BV_WORDS ((1u << 19) + 32u) /* INITIALBITARRAYSIZE, cu:68 */
#define ORC_MAX_LIMBS 16                 /* 512-bit values */

typedef struct {
  uint32_t maxbits;   /* N  (MAXBITS, cu:43) */
  uint32_t mbi;       /* N - A (MAXBITSINITIAL, cu:65) */
  uint32_t tpo;       /* THREEPOWEROFFSET, cu:67 */
  uint32_t magic[16]; /* cu:122-128 */
  uint32_t *bv;       /* 16 x ORC_BV_WORDS (initialbitarray, cu:77) */
  uint32_t mod9[9][32];
} orc_tables;

typedef struct {
  uint32_t hash;          /* "Complete hash" (cu:182) */
  uint64_t seeds;         /* surviving seeds iterated (sum of alength) */
  uint64_t pairs;         /* Step-1 leaves with bigindex < 16 */
  uint64_t cpu_pairs;     /* Step-1 leaves with bigindex >= 16 (cu:517) */
  uint64_t launches;      /* reference launchkernel calls (cu:181) */
  uint64_t checkpoints;   /* loop iterations of the Step-3 while(true) */
  uint64_t n_overflow;    /* seeds that reached 2^CUTOFFPOWER */
  uint64_t *overflow;     /* caller buffer of (lo, hi) pairs, may be NULL */
  uint64_t overflow_cap;  /* in seeds */
  uint64_t max_exc[2];    /* 128-bit values as (lo, hi) */
  uint64_t max_exc_seed[2];
  uint64_t max_st;
  uint64_t max_st_seed[2];
  uint64_t seeds_done;    /* seeds that entered the maxima (no overflow) */
} orc_case_result;

typedef struct {
  uint64_t seeds;        /* seeds iterated */
  uint64_t failures;     /* seeds whose value left 512 bits */
  uint32_t max_exc[ORC_MAX_LIMBS];
  uint32_t max_exc_seed[4];
  uint64_t max_st;
  uint32_t max_st_seed[4];
  uint64_t steps;        /* T-steps executed from the seed */
  uint64_t odd_runs, even_runs;
  uint64_t wide64;       /* method 3: seeds whose value left 64 bits (re-run in 128) */
} orc_range_result;

/* ---------------- cases mode (reference restatement) ---------------- */
int orc_tables_init(orc_tables *t, uint32_t maxbits);
void orc_tables_free(orc_tables *t);
void orc_case_result_init(orc_case_result *r);

/* Step 2 + Step 3 for one Step-1 pair.  cpu_sem = 0: compute_kernel
 * semantics (cu:185-411); cpu_sem = 1: search2/search3 semantics
 * (cu:654-715; used by the reference for bigindex >= 16).  Returns the
 * XOR hash contribution and accumulates into r. */
uint32_t orc_pair(const orc_tables *t, uint32_t bigindex, uint64_t base_lo,
                  uint64_t base_hi, uint64_t number_lo, uint64_t number_hi,
                  int cpu_sem, orc_case_result *r);

/* One whole reference run from a stdin 6-tuple (cu:95-183).  Returns 0,
 * or -1 when sigfig > N - A (the reference would recurse forever). */
int orc_run_case(const orc_tables *t, uint64_t base_lo, uint64_t base_hi,
                 uint32_t sigfig, uint32_t threepower, uint64_t number_lo,
                 uint64_t number_hi, uint32_t doubleeven, uint32_t numevens,
                 orc_case_result *r);

/* Step-1 leaves only (no Step 2/3): calls cb for every leaf in the
 * reference's visiting order. */
typedef void (*orc_leaf_cb)(void *ctx, uint32_t bigindex, uint64_t base_lo,
                            uint64_t base_hi, uint64_t number_lo,
                            uint64_t number_hi);
int orc_search1(const orc_tables *t, uint64_t base_lo, uint64_t base_hi,
                uint32_t sigfig, uint32_t threepower, uint64_t number_lo,
                uint64_t number_hi, uint32_t doubleeven, uint32_t numevens,
                orc_leaf_cb cb, void *ctx);

/* Step-1 subtree roots at a cut depth (used to split a case into
 * independent sub-cases, like the reference's cases_* files). */
typedef void (*orc_root_cb)(void *ctx, uint64_t base_lo, uint64_t base_hi,
                            uint32_t sigfig, uint32_t threepower,
                            uint64_t number_lo, uint64_t number_hi,
                            uint32_t doubleeven, uint32_t numevens);
int orc_split(const orc_tables *t, uint64_t base_lo, uint64_t base_hi,
              uint32_t sigfig, uint32_t threepower, uint64_t number_lo,
              uint64_t number_hi, uint32_t doubleeven, uint32_t numevens,
              uint32_t cut_sigfig, orc_root_cb cb, void *ctx);

/* ---------------- range mode ---------------- */
/* Sieve over residues r mod 2^k: bit r set iff 3^{f_j(r)} > 2^j for all
 * 1 <= j <= k (r cannot be shown to drop within k steps).  bits must hold
 * 2^k / 8 bytes.  Returns the number of survivors. */
uint64_t orc_range_sieve(uint32_t k, uint8_t *bits);
/* For every removed residue r, checks T^tau(2^k + r) < 2^k + r where tau
 * is the first j with 3^{f_j} < 2^j; by monotonicity this proves the
 * sieve for every n >= 2^k.  Returns the number of violations. */
uint64_t orc_range_sieve_validate(uint32_t k);

/* Range verification.  Seeds: n in [offset, offset+size), n >= 2, n mod 9
 * in {0,1,3,6,7} (when use_mod9), and, when n >= 2^k, r = n mod 2^k a
 * sieve survivor (k = 0: no residue sieve).  method 0 = single T-steps,
 * 1 = run-length loop after search3 (cu:684-715), 2 = the GPU kernel's
 * structure (one k-step jump, then method 1; counts runs after the jump),
 * 3 = method 1 in 64-bit unsigned arithmetic with overflow detection
 * (__builtin_mul_overflow on each odd run's multiply; a seed whose value
 * would leave 64 bits is re-run with method 1 and counted in wide64) -- the
 * plain CPU verification of n < 2^32 with 64-bit values.
 * All methods give identical results.  nthreads >= 1. */
int orc_range(uint64_t offset_lo, uint64_t offset_hi, uint64_t size,
              uint32_t k, int use_mod9, int method, int nthreads,
              orc_range_result *out);
/* As orc_range, with flags:
 *   ORC_RANGE_DIRECT_SIEVE -- test each seed's residue against the sieve's
 *     definition instead of building the 2^k-bit table (what orc_range does
 *     for k > 26 and for ranges much smaller than 2^k).  Same results.
 *   ORC_RANGE_NEGATIVE -- the negative-integer variant: seed m stands for
 *     -m and the map is T'(m) = (3m-1)/2 for odd m, m/2 for even m (T on
 *     -m).  The k-step sieve uses T's parity steps with the same descent
 *     test; the mod-9 sieve keeps m mod 9 in {0,2,3,6,8} (and m = 5), the
 *     analogue of {0,1,3,6,7} for T.  A seed that returns to itself (the
 *     cycle minima 5 and 17) or runs 2^22 steps without descending counts
 *     as a failure and enters neither maximum. */
#define ORC_RANGE_DIRECT_SIEVE 0x1
#define ORC_RANGE_NEGATIVE 0x2
int orc_range_ex(uint64_t offset_lo, uint64_t offset_hi, uint64_t size,
                 uint32_t k, int use_mod9, int method, int nthreads,
                 int flags, orc_range_result *out);

/* ---------------- trajectory queries ---------------- */
/* seeds: nseeds x seed_limbs little-endian u32 limbs (seed_limbs <= 8).
 * st: stopping time per seed; exc: 16 u32 limbs per seed; status: 0 ok,
 * 1 trivial (n < 2: no stopping time), 2 overflow (left 512 bits). */
int orc_trajectory(const uint32_t *seeds, uint32_t nseeds,
                   uint32_t seed_limbs, uint64_t *st, uint32_t *exc,
                   uint32_t *status);

#ifdef __cplusplus
}
#endif
#endif
