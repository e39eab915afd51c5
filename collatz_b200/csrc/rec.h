// rec.h -- per-request result record shared by device code and the host
// runtime (same layout on both sides).  One record accumulates one
// verification request: a reference case / pair batch, or one range.
#pragma once
#include <stdint.h>

namespace cz {

// error bits in ReqRec::errors
enum : uint32_t {
  ERR_LOCK = 1u << 0,        // a record lock was not acquired within its spin limit
  ERR_ITER_CAP = 1u << 1,    // a seed exceeded the per-seed iteration cap
  ERR_WIDEN_FULL = 1u << 2,  // the widening list overflowed
  ERR_SEED_SMALL = 1u << 3,  // a cases-mode seed < 3 (never descends, cu:362-368)
  ERR_OVERFLOW_CAP = 1u << 4 // more overflow seeds than the report buffer holds
};

struct ReqRec {
  unsigned long long seeds;       // seeds iterated
  unsigned long long st_key;      // running max stopping time (prefilter)
  unsigned long long e_key;       // monotone key of the running max excursion (prefilter)
  unsigned long long failures;    // seeds that did not finish (beyond widest limbs / iteration cap)
  unsigned long long widened;     // seeds re-run with wider limbs
  unsigned long long items_done;  // work items completed (serving progress); cases line batches: overflow reports
  uint32_t lock;                  // guards the exact maxima below
  uint32_t valid;                 // bit0: st fields set, bit1: E fields set
  uint32_t hash;                  // cases mode: XOR of all checkpoint low limbs (cu:359, 407-409)
  uint32_t errors;                // ERR_* bits
  unsigned long long st;          // exact maximum stopping time
  uint32_t st_seed[4];            // its seed (smallest on ties)
  uint32_t E[8];                  // exact maximum excursion (little-endian limbs)
  uint32_t E_seed[4];             // its seed (smallest on ties)
};
static_assert(sizeof(ReqRec) == 136, "ReqRec layout");

}  // namespace cz
