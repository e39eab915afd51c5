// kernels.h -- argument blocks and launchers of the hot-path kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rec.h"
#include "tables.h"

namespace cz {

// ---------------- cases mode (cases.cu) ----------------
struct CasesArgs {
  const uint32_t* pairs;   // npairs x 8 words: base limbs 0..3, number limbs 0..3 (cu:521-528)
  uint32_t npairs;
  int bigindex;            // >= 0: bucket of every pair; < 0: per pair in base limb 3
  const uint32_t* bv;      // CaseTables
  const uint32_t* mod9;
  const uint32_t* magic;
  const uint32_t* pow3;
  uint32_t mbi, tpo;
  uint32_t* pair_counter;  // scratch, zero before launch
  ReqRec* rec;
  uint32_t* overflow;      // overflow seeds, 4 words each
  uint32_t overflow_cap;
  unsigned long long* overflow_count;
  uint32_t iter_cap;       // checkpoints per seed before ERR_ITER_CAP
  uint32_t multi;          // line batch: base limb 3 = bigindex | line << 8, rec[line] per line
};
int cases_variants();
cudaError_t launch_cases(const CasesArgs& a, int variant, uint32_t grid, cudaStream_t st);
cudaError_t cases_occupancy(int variant, int* blocks_per_sm, bool multi = false);

// ---------------- device Step 1 (step1_dev.cu) ----------------
// A node of search1's tree (cu:497-505): base and number as little-endian
// 64-bit halves; sigfig | line << 8 (line: the node's cases line in a line
// batch), threepower, doubleeven, numevens.
struct S1Node {
  unsigned long long base_lo, base_hi, num_lo, num_hi;
  uint32_t sig, tp, de, ne;
};
static_assert(sizeof(S1Node) == 48, "S1Node layout");

// Counters of one device Step 1 run (zeroed before it starts).
struct S1Scalars {
  uint32_t level[128];  // frontier size after each breadth-first level
  uint32_t cursor[32];  // [0] count pass, [1 + chunk % 31] emit passes
  unsigned long long total;
  unsigned long long hist[17];  // leaves per bigindex; [16] = bigindex >= 16
};

struct Step1Args {
  uint32_t mbi, tpo;
  const S1Node* in;          // frontier
  const uint32_t* in_count;  // its size (device)
  S1Node* out;               // expand: children
  uint32_t* out_count;
  unsigned long long* off;   // walk: per frontier node, first leaf index
  unsigned long long* cnt;   // walk: per frontier node, leaves
  unsigned long long* total;
  unsigned long long* hist;
  unsigned long long* hist_lines;  // line batches: leaves per (line, bigindex), 17 per line; else null
  uint32_t* cursor;          // walk: zero before the launch
  ulonglong2* stk_num;       // walk: pending siblings, [level][thread]
  uint4* stk_meta;
  uint32_t nthreads;         // walk: threads of the launch (grid x 128)
  uint32_t* pairs;           // emit: pairs with leaf index in [w_lo, w_hi)
  unsigned long long w_lo, w_hi;
};
constexpr uint32_t STEP1_WALK_BLOCKS_PER_SM = 8;
cudaError_t launch_step1_expand(const Step1Args& a, uint32_t bound, cudaStream_t st);
cudaError_t launch_step1_walk(const Step1Args& a, bool emit, cudaStream_t st);

// ---------------- range mode (range.cu) ----------------
constexpr uint32_t RANGE_ITEM = 64;     // survivor-table entries per work item
constexpr uint32_t DENSE_ITEM = 64;     // consecutive integers per dense work item

// A run of work items of one request.  kind 0: survivor entries
// [s_lo, s_hi) (one mod-9 class of the class-major table, or all of it) of
// blocks q, q + qstride, ... (nq blocks; seeds n = q 2^k + r);
// kind 1: integers [d_lo, d_hi) iterated without the residue sieve.
struct RangeSeg {
  unsigned long long item_begin;  // global index of the first item
  unsigned long long q_lo;        // kind 0: first block, low 64 bits; kind 1: d_lo
  unsigned long long d_hi;        // kind 1: end (exclusive)
  uint32_t q_hi;                  // kind 0: first block, bits 64..95
  uint32_t nq;                    // kind 0: number of blocks
  uint32_t s_lo, s_hi;            // kind 0: survivor index range
  uint32_t ipq;                   // kind 0: items per block
  uint32_t req;                   // request index (ReqRec)
  uint16_t kind;
  uint16_t qstride;               // kind 0: block stride (0 or 1: consecutive blocks; 9: one q mod 9)
  uint32_t mod9;                  // 1: apply the mod-9 sieve to each entry (0 when the segment's
                                  //    classes are all kept by it)
  // Item index within the original segment of item_begin (non-zero when a
  // scheduler cuts a segment into slices; local indices stay < 2^32 for kind 0).
  uint32_t local0_lo, local0_hi;
};
static_assert(sizeof(RangeSeg) == 64, "RangeSeg");

struct WidenEntry {  // a seed to re-run with wider limbs
  uint32_t req, n0, n1, n2;
};

struct RangeArgs {
  const RangeEntry* table;        // survivor table of the 2^k sieve
  uint32_t k;
  const RangeSeg* segs;
  uint32_t nsegs;
  unsigned long long* item_cursor;  // scratch: next item to claim
  unsigned long long item_limit;    // items >= limit are not claimed in this launch
  ReqRec* recs;
  WidenEntry* widen;
  uint32_t widen_cap;
  uint32_t* widen_count;
  uint32_t iter_cap;              // odd/even run pairs per seed before ERR_ITER_CAP
  uint32_t negative;              // 1: the negative-integer variant (a table built for it)
  unsigned long long* stats;      // diagnostics counters (stats variant only), may be null
  uint32_t seed_bits;             // bit length of the launch's largest seed (0: not known)
};
// Variants 4 and 5 run the 64-bit body (variants 6 and 7) when every seed of
// the launch lies below 2^RANGE_NARROW_MAX_BITS: its values then stay below
// 2^59 for most steps.  For seeds from 2^52 on, the 128-bit body alone is
// faster (measured on B200: 2^34 seeds at 2^51 take 5.20 ms with the 64-bit
// body and 5.21 ms without; at 2^52, 5.29 ms and 5.21 ms).
constexpr uint32_t RANGE_NARROW_MAX_BITS = 52;
int range_variants();
cudaError_t range_init();  // once per device, before the first launch
// Diagnostics variant (the default shape with 3 blocks per SM): counts run
// pairs, slow paths, replays, jumps, pops, expansions, pop-block passes and
// offers into a.stats[0..7], clock64 cycles per phase into [8..13], 8-step
// windows taken into [14] and run pairs on the 64-bit body into [15].
cudaError_t launch_range_stats(const RangeArgs& a, uint32_t grid, cudaStream_t st);
cudaError_t launch_range(const RangeArgs& a, int variant, uint32_t grid, cudaStream_t st);
cudaError_t range_occupancy(int variant, int* blocks_per_sm);
// The 64-bit range kernel (range64.cu): the same seeds and results as
// launch_range for launches of the positive variant whose seeds all lie
// below 2^range64_max_seed_bits(); one 64-bit value per seed, four limbs per
// lane only while a lane's value is at or above 2^59.  Variants differ in
// run pairs per pass, resident blocks per SM and the in-loop table steps J
// (0: none; 8, 10, 11).
int range64_variants();
// Hash of the 64-bit kernel's variant table (part of the autotuner's cache key).
uint32_t range64_variant_rev();
uint32_t range64_max_seed_bits();
cudaError_t range64_init();  // once per device, before the first launch
cudaError_t launch_range64(const RangeArgs& a, int variant, uint32_t grid, cudaStream_t st);
// Diagnostics form: run pairs, slow paths, replays, jumps, pops, expansions,
// passes, offers into a.stats[0..7], table steps [13], windows [14], 64-bit
// pairs [15]; clock64 cycles of offers, refill and lanes into [8..10].
cudaError_t launch_range64_stats(const RangeArgs& a, int variant, uint32_t grid, cudaStream_t st);
cudaError_t range64_occupancy(int variant, int* blocks_per_sm);
// Threshold scouts: first_seg[i] is the index of request i's first segment
// (>= a.nsegs: none).  Raises each request's prefilter keys to the maxima of
// the seeds of its first work item, before the range kernel runs.
cudaError_t launch_range_scout(const RangeArgs& a, const uint32_t* first_seg, uint32_t nreq, cudaStream_t st);
// Seeds of a widen list re-run from scratch with 6 (then 8) limbs; the
// list length is read on the device (*count, at most cap), so the pass can
// sit in a captured graph right behind the range kernel.
cudaError_t launch_range_wide(const WidenEntry* list, const uint32_t* count, uint32_t cap, int limbs,
                              ReqRec* recs, WidenEntry* next, uint32_t next_cap, uint32_t* next_count,
                              uint32_t iter_cap, cudaStream_t st, bool negative = false);

// ---------------- trajectory queries (traj.cu) ----------------
// All limb classes in one launch (traj.cu): index = the seed ids sorted by
// limb class (4, 6, 8, 12, 16 limbs; class j at [cstart[j], cstart[j + 1])),
// one cursor (zero before the launch); a seed that needs more limbs is run
// again by the same thread with the next width.
struct TrajAllArgs {
  const uint32_t* seeds;       // nseeds x 8 limbs
  const uint32_t* index;       // cstart[5] entries
  uint32_t cstart[6];
  unsigned long long* st;      // out: stopping time
  uint32_t* exc;               // out: 16 limbs each
  uint32_t* status;            // out: 0 ok, 1 trivial, 2 overflow, 3 iteration cap
  uint32_t* cursor;            // scratch
  uint32_t iter_cap;
};
cudaError_t launch_traj_all(const TrajAllArgs& a, uint32_t grid, cudaStream_t st);
// Limb class of a seed of at most 256 bits (8 little-endian limbs): 0..4 for
// 4, 6, 8, 12, 16 limbs, leaving room for the value to grow before it is
// handed on.
inline uint32_t traj_class(const uint32_t* w) {
  uint32_t bl = 0;
  for (int j = 7; j >= 0; j--)
    if (w[j]) {
      bl = 32u * j + (32u - __builtin_clz(w[j]));
      break;
    }
  return bl <= 96 ? 0 : bl <= 160 ? 1 : bl <= 224 ? 2 : bl <= 352 ? 3 : 4;
}

}  // namespace cz
