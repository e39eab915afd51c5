// tables.h -- device-resident sieve tables (built on the GPU by tables.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cz {

constexpr uint32_t POW3_COUNT = 96;          // 3^f mod 2^128 for f < 96
constexpr uint32_t RANGE_CHUNK_WORDS = 1024; // sieve words per compaction chunk

// Cases mode (reference Algorithm 1, Steps 2-3).
struct CaseTables {
  uint32_t maxbits = 0, mbi = 0, tpo = 0;
  uint32_t* bv = nullptr;     // 16 x BV_WORDS, the reference's flat layout (cu:138-143)
  uint32_t* mod9 = nullptr;   // 9 x 32 (cu:159-164)
  uint32_t* magic = nullptr;  // 16
  uint32_t* pow3 = nullptr;   // POW3_COUNT x 4 limbs
};

// One surviving residue r mod 2^k (16 bytes).
//   r      = r_lo | (meta & 0xFF) << 32
//   f      = (meta >> 8) & 0xFF     odd steps among the first k
//   r mod 9 = (meta >> 16) & 0xFF
//   emax   = meta >> 24             max over j <= k of ceil(log2(3^f_j / 2^j)), >= 0
//   c      = c_lo | c_hi << 32      T^k(r) + 1
// so that for n = q 2^k + r:  T^k(n) + 1 = q 3^f + c.
struct RangeEntry {
  uint32_t r_lo, meta, c_lo, c_hi;
};
static_assert(sizeof(RangeEntry) == 16, "RangeEntry");

// The survivor table is class-major: the survivors with r = 0 mod 9 in
// residue order, then those with r = 1 mod 9, and so on.  For a block q the
// mod-9 sieve keeps n = q 2^k + r iff (q 2^k + r) mod 9 is in {0,1,3,6,7},
// which depends only on q mod 9 and r mod 9; so a block's seeds are 5 whole
// classes, and a work item (64 consecutive entries of one class) holds only
// seeds -- no entry is loaded and then dropped by the mod-9 sieve.
struct RangeTable {
  uint32_t k = 0;
  uint32_t* bits = nullptr;         // 2^k bits
  RangeEntry* table = nullptr;      // survivors, class-major (see above)
  unsigned long long count = 0;     // number of survivors
  unsigned long long cls[10] = {};  // class c = table[cls[c], cls[c+1])
  unsigned long long violations = 0;// sieve validation failures (must be 0)
  bool negative = false;            // built for the negative-integer variant
};

cudaError_t build_case_tables(CaseTables* t, uint32_t maxbits, cudaStream_t st);
void free_case_tables(CaseTables* t);
// negative: the sieve and jumps of the negative-integer variant T'(m) = (3m-1)/2, m/2 (the
// entries then hold c = T'^k(r) - 1, so that T'^k(n) - 1 = q 3^f + c).
cudaError_t build_range_table(RangeTable* t, uint32_t k, bool validate, cudaStream_t st, bool negative = false);
void free_range_table(RangeTable* t);

}  // namespace cz
