/*
 * collatz.h -- C ABI of collatz_b200, a B200-native (sm_100a) Collatz
 * convergence verifier with the inputs and outputs of the reference
 * program collatz_cudav7.cu (vigleik0/collatz).
 *
 * Conventions: every entry point returns an int status (COLLATZ_OK = 0,
 * negative on error) and never throws.  The caller owns every host buffer;
 * the library owns its device memory (sieve tables, scratch).  Numbers
 * wider than 64 bits are little-endian arrays of uint64_t (u128 fields) or
 * uint32_t limbs.  A context is used by one host thread at a time (calls
 * on one context are serialised internally); the server object is the
 * thread-safe front end.
 *
 * Definitions (T is the reference's shortcut map, main.rs:13):
 *   T(n) = (3n+1)/2 for odd n, n/2 for even n.
 *   stopping time  sigma(n) = least k >= 1 with T^k(n) < n.
 *   excursion      E(n) = max over 0 <= k <= sigma(n) of T^k(n).
 * In cases mode Step 1 carries no per-seed history, so E is the maximum
 * over N-A <= k <= sigma(n); sigma still counts from n.  Ties in either
 * maximum go to the smaller seed.
 */
#ifndef COLLATZ_B200_H
#define COLLATZ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define COLLATZ_ABI_VERSION 2

enum collatz_status_code {
  COLLATZ_OK = 0,
  COLLATZ_E_ARG = -1,       /* invalid argument */
  COLLATZ_E_CUDA = -2,      /* CUDA runtime error (see collatz_last_error) */
  COLLATZ_E_NOMEM = -3,     /* host or device allocation failed */
  COLLATZ_E_LIMIT = -4,     /* request beyond a documented size limit */
  COLLATZ_E_DEVICE = -5,    /* a kernel reported an error bit (see result.errors) */
  COLLATZ_E_TIMEOUT = -6,   /* poll timed out */
  COLLATZ_E_STATE = -7,     /* object in the wrong state (e.g. server stopped) */
  COLLATZ_E_ADMISSION = -8, /* request refused: not enough free device memory */
  COLLATZ_E_NODEV = -9      /* no CUDA device / the kernels are not loadable */
};

/* device error bits reported in result.errors */
#define COLLATZ_ERR_LOCK 0x1u        /* a result lock spin hit its limit */
#define COLLATZ_ERR_ITER_CAP 0x2u    /* a seed exceeded the per-seed iteration cap */
#define COLLATZ_ERR_WIDEN_FULL 0x4u  /* widening list full */
#define COLLATZ_ERR_SEED_SMALL 0x8u  /* cases mode: a seed < 3 (never descends) */

typedef struct collatz_ctx collatz_ctx;

typedef struct {
  uint32_t maxbits;     /* N = MAXBITS (collatz_cudav7.cu:43); 16..96; default 45 */
  uint32_t range_k;     /* default residue-sieve exponent of range requests; default 24 */
  int32_t device;       /* CUDA device ordinal; default 0 */
  uint32_t variant;     /* kernel variant, COLLATZ_VARIANT_AUTO = tuned default */
  uint32_t iter_cap;    /* per-seed loop cap in checkpoints / run pairs (0 = default 1<<16) */
  uint32_t flags;       /* COLLATZ_CFG_* bits; default 0 */
  uint32_t reserved[10];
} collatz_config;
#define COLLATZ_VARIANT_AUTO 0xFFFFFFFFu
/* collatz_run_case runs Step 1 (search1, cu:497-563) on the host threads
 * and copies the pairs to the device, instead of on the device. */
#define COLLATZ_CFG_HOST_STEP1 0x1u

void collatz_config_default(collatz_config *cfg);
/* Builds the reference's sieve tables for cfg->maxbits on the device
 * (replaces precompute, cu:423-495, and the uploads of cu:133-171). */
int collatz_create(const collatz_config *cfg, collatz_ctx **out);
void collatz_destroy(collatz_ctx *ctx);
const char *collatz_status_string(int status);
const char *collatz_last_error(const collatz_ctx *ctx);
/* Work is issued on this CUDA stream (cudaStream_t; NULL = the library's
 * own stream). */
int collatz_set_stream(collatz_ctx *ctx, void *cuda_stream);
int collatz_device_info(const collatz_ctx *ctx, int *sm_count, int *sm_clock_khz);

/* ------------------------------------------------------------------ */
/* Cases mode: the reference's verification run (Algorithm 1).         */
/* ------------------------------------------------------------------ */

/* One stdin line of the reference: "base sigfig threepower number
 * doubleeven numevens" (cu:96-101, 174), the format of cases_*. */
typedef struct {
  uint64_t base[2];
  uint32_t sigfig;
  uint32_t threepower;
  uint64_t number[2];
  uint32_t doubleeven;
  uint32_t numevens;
} collatz_case;

typedef struct {
  uint32_t hash;            /* "Complete hash" (cu:182) */
  uint32_t spot_checks;     /* always 0: the product never recomputes on the CPU */
  uint64_t launches;        /* the reference's "Number of kernel launches" (cu:181) */
  uint64_t seeds_checked;   /* surviving seeds iterated */
  uint64_t pairs;           /* Step-1 leaves with bigindex < 16 */
  uint64_t cpu_pairs;       /* Step-1 leaves with bigindex >= 16 (cu:517-519), run on the GPU */
  uint64_t n_overflow;      /* seeds whose value reached 2^100 (the reference prints them) */
  uint32_t *overflow_seeds; /* caller buffer: 4 uint32_t limbs per seed, sorted ascending; may be NULL */
  uint64_t overflow_cap;    /* capacity of overflow_seeds, in seeds */
  uint32_t max_excursion[4];
  uint32_t max_excursion_seed[4];
  uint64_t max_stopping_time;
  uint32_t max_stopping_time_seed[4];
  uint32_t errors;          /* COLLATZ_ERR_* bits */
  uint32_t reserved;
  double device_ms;         /* device time of the kernels (Steps 2/3, and Step 1 when on the device) */
} collatz_case_result;

/* Whole run from one 6-tuple (replaces main, cu:95-183).  Step 1
 * (search1, cu:497-563) runs on the device and writes the pairs into
 * device memory, where Steps 2-3 read them; with COLLATZ_CFG_HOST_STEP1 it
 * runs on all host threads feeding batches to the GPU instead.  Both give
 * the same result. */
int collatz_run_case(collatz_ctx *ctx, const collatz_case *c, collatz_case_result *out);

/* No counterpart in the reference.  Runs cases[0..n) together
 * (n <= COLLATZ_CASE_BATCH_MAX): the lines at least 20 levels above the
 * leaves (N - A - sigfig >= 20, each enough to fill the GPU) run one after
 * another as in collatz_run_case; all the others share one device pass:
 * Step 1 from all their roots at once, then Steps 2-3 with a record per
 * case.  For a file of many small lines (cases_big) this replaces n calls of
 * collatz_run_case, whose fixed cost per call would dominate.  out[i] receives what collatz_run_case gives
 * for cases[i]: hash, launches, seeds, pairs, maxima, errors, n_overflow;
 * device_ms is the pass's device time split by seeds.  Overflow seeds go to
 * one pool (4 uint32 per seed, pool_cap seeds), grouped by case, ascending
 * within a case: out[i].overflow_seeds / overflow_cap are set to case i's
 * part of the pool (NULL / 0 when it has none or the pool is full).  At most
 * 65536 overflow seeds are kept per call; n_overflow counts all of them. */
#define COLLATZ_CASE_BATCH_MAX (1u << 20)
int collatz_run_case_batch(collatz_ctx *ctx, const collatz_case *cases, uint32_t n, collatz_case_result *out,
                           uint32_t *overflow_pool, uint64_t pool_cap);

/* One batch of Step-1 pairs of one bucket (replaces launchkernel,
 * cu:565-649, and compute_kernel, cu:185-411).  pairs: npairs x 8 uint32
 * (base limbs 0..3, number limbs 0..3; base limb 3 is ignored as in
 * cu:201).  bigindex = threepower - THREEPOWEROFFSET; bigindex >= 16 runs
 * search2/search3 semantics (cu:654-715).  The result accumulates nothing
 * across calls. */
int collatz_verify_pairs(collatz_ctx *ctx, uint32_t bigindex, const uint32_t *pairs, uint32_t npairs,
                         collatz_case_result *out);

/* No counterpart in the reference.  collatz_verify_pairs for callers that
 * cannot allocate memory while they verify: an application that gives this
 * library device buffers from its own memory pool and allows no other
 * allocation, or a latency-bound loop in which cudaMalloc/cudaFree, which can
 * block and synchronize the device, are not allowed.  It allocates nothing:
 * d_pairs (npairs x 8 uint32, same layout as collatz_verify_pairs) is
 * already in device memory, the result comes back in *out (host), and the
 * kernel's scratch is a fixed 64 KiB device array that every GPU loading the
 * library holds until exit.  At most 4064 overflow seeds are reported per
 * call: out->overflow_cap above 4064 is rejected with COLLATZ_E_LIMIT (when
 * more seeds overflow than are reported, n_overflow still counts all of
 * them).  The first call on a device looks up the array's device address;
 * make that first call before any stream capture.  Calls share the array,
 * so calls that overlap on the GPU race; the context's mutex serialises
 * calls made through one context. */
int collatz_verify_pairs_noalloc(collatz_ctx *ctx, uint32_t bigindex, const uint32_t *d_pairs,
                                 uint32_t npairs, collatz_case_result *out);

/* Step-1 leaves of a case (search1, cu:497-563) for N = maxbits, in the
 * reference's order, without Steps 2-3: each pair as 8 uint32 with base
 * limb 3 = bigindex.  *count receives the number of leaves (pairs are
 * written up to cap).  Host-only: needs no device. */
int collatz_step1_pairs(uint32_t maxbits, const collatz_case *c, uint32_t *pairs, uint64_t cap,
                        uint64_t *count);

/* No counterpart in the reference (its cases_* files are cut this way).
 * The nodes of a case's Step-1 tree at sigfig = cut, c->sigfig <= cut <=
 * N - A, i.e. the roots of search1's subtrees there (cu:497-563), in the
 * reference's visiting order, as 6-tuples: run as cases, the XOR of their
 * hashes and the sums of their counts equal the whole case's.  *count
 * receives the number of nodes; cases are written up to cap.  Host-only. */
int collatz_step1_split(uint32_t maxbits, const collatz_case *c, uint32_t cut, collatz_case *out, uint64_t cap,
                        uint64_t *count);

/* No counterpart in the reference.  The Step-1 leaves of a case computed by
 * the device Step 1 of collatz_run_case, for the context's N, in no
 * particular order (the same multiset as collatz_step1_pairs).  *count
 * receives the number of leaves; pairs (8 uint32 each, base limb 3 =
 * bigindex) are written up to cap. */
int collatz_step1_pairs_device(collatz_ctx *ctx, const collatz_case *c, uint32_t *pairs, uint64_t cap,
                               uint64_t *count);

/* ---- Cases driver: many cases_* lines with a resume journal ---- */
/* The reference is run as one process per cases_* line and the results are
 * combined by hand (multi-copy operation).  These calls do it in one process.
 *
 * Merges per-case results: hash by XOR, counts and device time by sum,
 * maxima by value then smaller seed, overflow seeds concatenated and sorted
 * (up to out->overflow_cap; n_overflow counts all), errors by OR.
 * Host-only. */
int collatz_combine_case_results(const collatz_case_result *parts, uint32_t n, collatz_case_result *out);

/* Runs cases[0..n) on one context, in groups of up to 8192 cases per
 * device pass (collatz_run_case_batch), and combines them into *combined.
 * With a journal path, each finished case is appended to the journal as one
 * text line; a group's lines are flushed and synced before the next group
 * starts.  A later call with the same cases and journal takes the finished
 * cases from the journal and runs only the rest, so an interrupted run
 * resumes where it stopped.  A journal line whose tuple differs from the case at its index is
 * rejected (COLLATZ_E_STATE).  per_case (NULL or n entries) receives each
 * case's result without overflow seeds.  *n_run (may be NULL) = cases run by
 * this call. */
int collatz_run_cases(collatz_ctx *ctx, const collatz_case *cases, uint32_t n, const char *journal,
                      collatz_case_result *per_case, collatz_case_result *combined, uint32_t *n_run);

/* Host-only: reads a journal.  For every case index it records, done[i] = 1
 * and results[i] receives that case's result; results[i].overflow_seeds is
 * filled up to results[i].overflow_cap when set.  A missing journal file
 * means nothing is done yet. */
int collatz_journal_load(const char *journal, const collatz_case *cases, uint32_t n,
                         collatz_case_result *results, uint8_t *done);

/* Copies the device-built tables back: bv = 16 x (2^19 + 32) uint32 (the
 * reference's flat d_flat, cu:138-152), mod9 = 9 x 32 uint32 (cu:159-171). */
int collatz_case_tables(collatz_ctx *ctx, uint32_t *bv, uint32_t *mod9);

/* ------------------------------------------------------------------ */
/* Range mode and trajectory queries (new entry modes).                */
/* ------------------------------------------------------------------ */

/* Seeds n in [offset, offset + size) with n >= 2 and, with the sieves on,
 * n mod 9 in {0,1,3,6,7} and (for n >= 2^k) n mod 2^k a survivor of the
 * k-step descent sieve.  offset + size <= 2^96, size <= 2^48, k in 8..34. */
typedef struct {
  uint64_t offset[2];
  uint64_t size;
  uint32_t k;      /* 0 = the context's range_k */
  uint32_t flags;  /* COLLATZ_RANGE_NO_MOD9, COLLATZ_RANGE_NEGATIVE */
} collatz_range;
#define COLLATZ_RANGE_NO_MOD9 0x1u
/* Negative integers (no counterpart in the reference): seed m stands for -m,
 * and the map is T'(m) = (3m-1)/2 for odd m, m/2 for even m (T acting on
 * -m).  The residue sieve uses T's parity steps with the same descent
 * test; the mod-9 sieve keeps m mod 9 in {0,2,3,6,8} (m = 1 mod 3 is T' of
 * the smaller (2m+1)/3, m = 5 mod 9 is T'^3 of the smaller (8m+5)/9) and
 * m = 5.  A seed that returns to itself never descends: the cycle minima 5
 * and 17 are reported in failures (no error bit).  Requests of one batch
 * or plan are all negative or all positive. */
#define COLLATZ_RANGE_NEGATIVE 0x2u

typedef struct {
  uint64_t seeds_checked;
  uint64_t failures;         /* seeds that did not finish within 256-bit values or the iteration cap */
  uint64_t widened;          /* seeds re-run with 192/256-bit values */
  uint32_t max_excursion[8]; /* 256-bit */
  uint32_t max_excursion_seed[4];
  uint64_t max_stopping_time;
  uint32_t max_stopping_time_seed[4];
  uint32_t errors;           /* COLLATZ_ERR_* bits */
  int32_t status;
  double device_ms;
} collatz_range_result;

int collatz_verify_range(collatz_ctx *ctx, const collatz_range *r, collatz_range_result *out);
/* Many requests in one persistent launch (device work queue). */
int collatz_verify_batch(collatz_ctx *ctx, const collatz_range *r, uint32_t n, collatz_range_result *out);

/* Device-resident form for timing: a plan holds the lowered work list on
 * the device and a captured CUDA graph (reset, kernel, widening passes). */
typedef struct collatz_plan collatz_plan;
int collatz_plan_create(collatz_ctx *ctx, const collatz_range *r, uint32_t n, collatz_plan **out);
int collatz_plan_launch(collatz_plan *p);   /* enqueue on the context stream, no sync */
int collatz_plan_results(collatz_plan *p, collatz_range_result *out); /* sync + copy back */
void collatz_plan_destroy(collatz_plan *p);

/* Copies the range-mode residue sieve for k back: bits (2^k / 8 bytes,
 * bit r set iff r mod 2^k survives) and the survivor count. */
int collatz_range_sieve(collatz_ctx *ctx, uint32_t k, uint8_t *bits, uint64_t *count);

/* Per-seed stopping time and excursion.  seeds: n x 8 uint32 limbs
 * (seeds < 2^256).  stopping_time[i]; excursion: 16 limbs (512 bits) per
 * seed; status[i]: 0 ok, 1 seed < 2 (no stopping time), 2 value left 512
 * bits, 3 iteration cap. */
int collatz_trajectory(collatz_ctx *ctx, const uint32_t *seeds, uint32_t n, uint64_t *stopping_time,
                       uint32_t *excursion, uint32_t *status);

/* ------------------------------------------------------------------ */
/* Serving (new entry mode): continuous batching of range requests and */
/* trajectory queries on one device.                                   */
/* ------------------------------------------------------------------ */
/* Worker threads admit requests in arrival order while request slots
 * and, for trajectory queries, free device memory allow (cudaMemGetInfo
 * minus hbm_reserve, read every 50 ms by a budget thread),
 * cuts the admitted range requests into slices of work items that share
 * one persistent range launch (small requests take what they need, the
 * rest of the slice goes to the large ones), runs trajectory queries as
 * concatenated batches on a second stream so both overlap on the device,
 * and completes each request as soon as its last slice or batch is done.
 * Every result is identical to the same request run alone. */
typedef struct collatz_server collatz_server;

enum { COLLATZ_REQ_RANGE = 0, COLLATZ_REQ_TRAJECTORY = 1 };

typedef struct {
  uint32_t max_active;        /* range requests admitted at once, and as many trajectory queries;
                               * default 256, at most 4096 */
  uint32_t slice_items;       /* work items (64 survivor entries) per range slice; default 1 << 19 */
  uint64_t hbm_reserve;       /* device bytes that admission leaves free; default 1 GiB */
  uint32_t traj_batch_seeds;  /* seeds per trajectory batch (and per query); default 1 << 20, at
                                 most 1 << 22; the server pins 2 x 128 bytes per batch seed */
  uint32_t reserved[7];
} collatz_server_config;

typedef struct {
  uint32_t kind;               /* COLLATZ_REQ_* */
  uint32_t nseeds;             /* trajectory: number of seeds (1 .. traj_batch_seeds) */
  collatz_range range;         /* range request */
  /* trajectory: nseeds x 8 uint32 limbs in, outputs as collatz_trajectory;
   * the caller keeps all four buffers alive until collatz_server_wait
   * has returned this request's response. */
  const uint32_t *seeds;
  uint64_t *stopping_time;
  uint32_t *excursion;
  uint32_t *status;
} collatz_request;

typedef struct {
  uint64_t ticket;
  int32_t status;              /* COLLATZ_OK, COLLATZ_E_ADMISSION, COLLATZ_E_DEVICE, ... */
  uint32_t kind;
  collatz_range_result range;  /* range requests */
  double submit_s, admit_s, done_s; /* server clock (seconds since start) */
} collatz_response;

typedef struct {
  uint64_t submitted, admitted, completed, refused;
  uint64_t range_slices, traj_batches;
  uint64_t range_seeds_checked, traj_seeds;
  uint32_t active, pending;
  uint64_t hbm_free;           /* cudaMemGetInfo free bytes at the last budget read */
  uint64_t hbm_admitted;       /* device bytes held by admitted requests */
  double device_busy_s;        /* summed device time of range slices */
  /* scheduler thread: loop iterations and host seconds spent admitting,
   * building slices, building batches, completing requests, and idle */
  uint64_t loops;
  double host_admit_s, host_slice_s, host_batch_s, host_complete_s, host_idle_s;
} collatz_server_info_t;

void collatz_server_config_default(collatz_server_config *scfg);
/* Creates a context for cfg->device (tables built and kept resident) and
 * starts the scheduler thread. */
int collatz_server_start(const collatz_config *cfg, const collatz_server_config *scfg, collatz_server **out);
/* Thread-safe.  Validates the request (COLLATZ_E_ARG / COLLATZ_E_LIMIT)
 * and queues it; *ticket identifies its response. */
int collatz_server_submit(collatz_server *s, const collatz_request *req, uint64_t *ticket);
/* Thread-safe.  Waits up to timeout_s (< 0: forever) for a ticket's
 * response, fills *resp and forgets the ticket.  Returns the request's
 * status, COLLATZ_E_TIMEOUT, or COLLATZ_E_ARG for an unknown ticket. */
int collatz_server_wait(collatz_server *s, uint64_t ticket, double timeout_s, collatz_response *resp);
int collatz_server_info(collatz_server *s, collatz_server_info_t *info);
/* Finishes the work on the device, fails queued requests with
 * COLLATZ_E_STATE, joins the scheduler and frees the server. */
int collatz_server_stop(collatz_server *s);

/* Kernel choices for the autotuner (no counterpart in the reference).
 *   COLLATZ_MODE_CASES, COLLATZ_MODE_RANGE: variant (block shape, body) of
 *     the cases kernel and of the four-limb range kernel;
 *   COLLATZ_MODE_RANGE64: variant of the 64-bit range kernel (jump-table
 *     window of 10 or 11 steps, run pairs at expansion, warp votes per step,
 *     queue-pop threshold, blocks per SM);
 *   COLLATZ_MODE_RANGE64_BITS: the limb width -- launches whose seeds all have
 *     at most this many bits (0..52) run the 64-bit kernel, the others the
 *     four-limb kernel (0: always four limbs).
 * collatz_variant_count gives the number of choices (0..count-1). */
#define COLLATZ_MODE_CASES 0
#define COLLATZ_MODE_RANGE 1
#define COLLATZ_MODE_RANGE64 2
#define COLLATZ_MODE_RANGE64_BITS 3
int collatz_variant_count(int mode);
int collatz_set_variant(collatz_ctx *ctx, int mode, int variant);

/* Autotuner (no counterpart in the reference).  Times every variant of the
 * selected modes on a fixed sample on this device and keeps the fastest:
 *   range: the four-limb kernel's variants and the 64-bit kernel's variants
 *     (window length j of the jump table, windows and run pairs per seed at
 *     expansion, in-loop table steps) on 2^34 seeds at 2^40 with the
 *     context's k, then the limb width: the two best variants timed on the
 *     2^32 largest seeds of 44 bits and of 48 bits; range64_bits is the
 *     largest of 48, 44 at which the 64-bit kernel is faster, else 0 (four
 *     limbs throughout);
 *   cases: about 2^20 Step-1 pairs of the root case "3 2 2 9 1 0" for the
 *     context's N.
 * The choices go into a text cache (COLLATZ_TUNE_CACHE, else
 * $XDG_CACHE_HOME/collatz_b200/tune.txt or ~/.cache/collatz_b200/tune.txt),
 * keyed by device, variant set and k or N.  A context created with
 * COLLATZ_VARIANT_AUTO applies cached choices; with COLLATZ_AUTOTUNE=1 in the
 * environment it also tunes what the cache lacks.  Variants and the limb
 * width never change results, only speed. */
typedef struct {
  int32_t range_variant, cases_variant; /* chosen (or kept when not tuned) */
  float range_ms[8], cases_ms[8];       /* device ms per variant on the sample; -1 = not timed */
  int32_t range64_variant;              /* 64-bit range kernel: chosen variant */
  uint32_t range64_bits;                /* chosen limb width (COLLATZ_MODE_RANGE64_BITS) */
  float range64_ms[8];                  /* device ms per 64-bit variant on the sample; -1 = not timed */
  float width_ms[4];                    /* 44-bit seeds: four limbs, 64 bits; 48-bit seeds: four limbs, 64 bits */
} collatz_tune_result;
#define COLLATZ_TUNE_RANGE 0x1u
#define COLLATZ_TUNE_CASES 0x2u
#define COLLATZ_TUNE_NO_CACHE 0x4u /* do not record the choice in the cache */
int collatz_autotune(collatz_ctx *ctx, uint32_t flags, collatz_tune_result *out);

/* Measured 32-bit integer peak of the context's device (no counterpart in
 * the reference; the roofline denominator of the integer-issue-bound
 * kernels).  Every SM runs 8 blocks of 256 threads, each thread 8
 * independent chains of dependent operations; the fastest of 3 timed
 * launches after a warm-up is kept.  mix 0: funnel shift, 3-input add and
 * 3-input logic op per link (ALU pipe only); mix 1: funnel shift, 3-input
 * add and multiply-add per link (two ALU operations to one FMA-pipe
 * multiply-add, the proportion of the run arithmetic).  About 0.2 s. */
typedef struct {
  uint64_t ops;          /* 32-bit operations of one launch */
  float ms;              /* its CUDA-event time */
  uint32_t mix, sm_count;
  double ops_per_s;      /* whole device */
  double sm_mhz;         /* SM clock during the launch (clock64 / global timer) */
  double ops_per_clk_sm; /* ops_per_s / (sm_mhz x sm_count): scales to other clocks */
} collatz_int_peak_t;
int collatz_int_peak(collatz_ctx *ctx, int mix, collatz_int_peak_t *out);

#ifdef __cplusplus
}
#endif
#endif /* COLLATZ_B200_H */
