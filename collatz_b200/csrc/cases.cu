// cases.cu -- reference-compatible Step 2 + Step 3 (collatz_cudav7.cu
// compute_kernel, cu:185-411; search2/search3, cu:654-715) for batches of
// Step-1 pairs.
//
// Design (B200): persistent warps.  A warp takes one pair at a time, reads
// the 33 look-ahead words of BV_f with one coalesced load per lane, ANDs
// the mod-9 row, and ranks the surviving high-bit values with popc + a warp
// scan into a per-warp queue in shared memory.  Lanes pull seeds from the
// queue as they finish, so a pair with 500 survivors no longer serialises
// in one thread (the reference runs one pair per thread).  Each lane runs
// the reference's checkpoint structure exactly -- [odd run <= 8, overflow
// test, even run <= 31] x 2, XOR the low limb, stop when v < n -- so the
// XOR hash, the seed count and the overflow list are identical; the order
// of work does not matter because every output is an XOR, a sum or a max.
// Stopping time and maximum excursion are tracked on the side.  While every
// lane running a step holds a value below 2^59, the step runs on one 64-bit
// value instead of four limbs (variant 4, for N <= 52).
//
// Line batches (MULTI): the pairs of many cases_* lines in one launch.  Base
// limb 3 of a pair holds bigindex | line << 8 and every line has its own
// record.  A pair slot keeps its line and that line's prefilter thresholds;
// a lane folds checkpoint XORs into a register for one line at a time and
// flushes it to the line's record when it takes a seed of another line; a
// warp counts seeds the same way.  Warps claim pairs 16 at a time, so
// neighbouring pairs (mostly one line's) stay on one warp.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"
#include "tables.h"

namespace cz {

constexpr u32 CQ = 1024;  // queue entries per warp (>= 31 + 570 survivors of one pair)
constexpr u32 CR = 32;    // pair slots per warp (a queue of < 32 entries spans < 32 pairs)
constexpr u32 CWARPS = 8;
constexpr u32 MULTI_CLAIM = 16;  // pairs per claim in line batches

template <bool MULTI>
struct CasesWarp {
  unsigned short q[CQ];             // (slot << 10) | a
  u32 ring[CR][MULTI ? 17 : 12];    // base0..2, number0..3, 3^f limbs 0..3, flags (bit 0 cpu, line << 1);
                                    // MULTI: [12] st threshold, [13..16] excursion threshold of the line
  u32 lane[32][MULTI ? 14 : 8];     // per lane: [0] st, [1..3] seed, [4..7] seed-local max E;
                                    // MULTI: [8] st threshold, [9..12] excursion threshold of its line,
                                    // [13] the line of a pending offer
  u32 thr[4];                       // excursion threshold (lower bound of the running max)
};

// Offers of several pending lanes (all lanes call this together; lane slots
// [0] sigma, [1..3] seed, [4..7] excursion, and in line batches [13] the
// line): a value that another pending lane of the same line beats -- larger,
// or equal with a smaller seed -- cannot be the line's maximum, so its bit is
// dropped.  A warp's first seeds of a line all finish under zero thresholds.
// Kept out of line: it runs in few passes.
template <int WD, bool MULTI>
__device__ __noinline__ u32 cases_drop_dominated(u32 (*L)[WD], u32 lane, u32 pend, u32 pm) {
  const u32 m1 = __ballot_sync(FULL, pend & 1u), m2 = __ballot_sync(FULL, pend & 2u);
  __syncwarp();
  if (pend) {
    const u32 s0 = L[lane][1], s1 = L[lane][2], s2 = L[lane][3];
    for (u32 m = pm & ~(1u << lane); m; m &= m - 1) {
      const u32 j = __ffs(m) - 1;
      if (MULTI && L[j][MULTI ? 13 : 0] != L[lane][MULTI ? 13 : 0]) continue;
      const u32 t0 = L[j][1], t1 = L[j][2], t2 = L[j][3];
      const bool j_smaller = (t2 != s2) ? (t2 < s2) : ((t1 != s1) ? (t1 < s1) : (t0 < s0));
      if ((pend & 1u) && ((m1 >> j) & 1u)) {
        const u32 sj = L[j][0], si = L[lane][0];
        if (sj > si || (sj == si && j_smaller)) pend &= ~1u;
      }
      if ((pend & 2u) && ((m2 >> j) & 1u)) {
        int c = 0;  // E_j against this lane's E, from the top limb
#pragma unroll
        for (int i = 7; i >= 4; i--)
          if (c == 0) c = (L[j][i] > L[lane][i]) ? 1 : ((L[j][i] < L[lane][i]) ? -1 : 0);
        if (c > 0 || (c == 0 && j_smaller)) pend &= ~2u;
      }
    }
  }
  __syncwarp();
  return pend;
}

// Exact excursion candidate x = v - 1 against the seed's maximum so far (or the
// threshold): kept as the seed's maximum when it is at least as large.
#define CASES_EXC_CANDIDATE()                                                                    \
  do {                                                                                           \
    const u32 x0 = v0 - 1, x1 = v1 - (v0 == 0), x2 = v2 - ((v0 | v1) == 0),                      \
              x3 = v3 - ((v0 | v1 | v2) == 0);                                                   \
    const u32* ref = evalid ? &W.lane[lane][4] : (MULTI ? &W.lane[lane][9] : W.thr);             \
    const bool ge = !lt96(x1, x2, x3, ref[1], ref[2], ref[3]) &&                                 \
                    !((x3 == ref[3]) & (x2 == ref[2]) & (x1 == ref[1]) & (x0 < ref[0]));         \
    if (ge) {                                                                                    \
      W.lane[lane][4] = x0;                                                                      \
      W.lane[lane][5] = x1;                                                                      \
      W.lane[lane][6] = x2;                                                                      \
      W.lane[lane][7] = x3;                                                                      \
      evalid = 1;                                                                                \
    }                                                                                            \
  } while (0)

template <int ITERS, int REFILL_MIN, bool MULTI, bool N64 = false>
__global__ void __launch_bounds__(CWARPS * 32) k_cases(const CasesArgs A) {
  __shared__ CasesWarp<MULTI> S[CWARPS];
  // 3^a for the 64-bit body: one shared load on the load/store pipe instead of
  // the ALU byte lookups (the ALU pipe is the busy one)
  __shared__ u32 s_p3[9];
  if (threadIdx.x < 9) {
    u32 p = 1;
    for (u32 i = 0; i < threadIdx.x; i++) p *= 3u;
    s_p3[threadIdx.x] = p;
  }
  const u32 lane = lane_id();
  CasesWarp<MULTI>& W = S[threadIdx.x >> 5];
  if (lane < 4) W.thr[lane] = 0;
  __syncthreads();

  const u32 mbi = A.mbi;
  // warp-uniform state
  u32 qhead = 0, qcount = 0, ring_seq = 0;
  bool exhausted = false;
  u32 thr_st = 0, thr3 = 0, thr2 = 0;
  ull warp_seeds = 0;
  u32 pc = 0, pc_end = 0;  // MULTI: claimed pairs [pc, pc_end)
  u32 wline = 0;           // MULTI: the line whose seeds warp_seeds counts
  // lane state
  bool active = false;
  u32 v0 = 0, v1 = 0, v2 = 0, v3 = 0, n0 = 0, n1 = 0, n2 = 0;
  u32 st = 0, iters = 0, hash = 0;
  u32 nbl = 0;  // bit length of the seed n
  u32 sig = 0;  // the stopping time, set at the first descent (st keeps counting)
  u32 found = 0, ovf = 0, cpu = 0, evalid = 0, pend = 0;
  u32 hline = 0;      // MULTI: the line whose checkpoint XORs `hash` holds (and of the lane's seed)
  u64 lthr_top = 0;   // MULTI: the lane's line's excursion threshold, bits 64..127

  for (;;) {
    // ---- offers of finished seeds, one lane at a time (bounded locks) ----
    {
      u32 pm = __ballot_sync(FULL, pend != 0);
      if (pm & (pm - 1)) {  // several pending lanes: offer only the best of each line
        pend = cases_drop_dominated<MULTI ? 14 : 8, MULTI>(W.lane, lane, pend, pm);
        pm = __ballot_sync(FULL, pend != 0);
      }
      while (pm) {
        const u32 leader = __ffs(pm) - 1;
        if (lane == leader) {
          u32 seed[4] = {W.lane[lane][1], W.lane[lane][2], W.lane[lane][3], 0};
          ReqRec* rec = MULTI ? A.rec + hline : A.rec;
          if (pend & 1u) rec_offer_st(rec, W.lane[lane][0], seed);
          if (pend & 2u) rec_offer_e<4>(rec, &W.lane[lane][4], seed);
          pend = 0;
        }
        pm &= pm - 1;
      }
      __syncwarp();
    }

    // ---- refill the queue and hand seeds to idle lanes ----
    const u32 idle = __ballot_sync(FULL, !active);
    const u32 nidle = __popc(idle);
    if (nidle >= (u32)REFILL_MIN || nidle == 32u) {
      while (qcount < nidle && !exhausted) {
        u32 p = 0;
        if (MULTI) {
          if (pc >= pc_end) {
            // 16 pairs per claim while many remain; single pairs for the tail
            const u32 claim =
                ((unsigned long long)pc + (unsigned long long)MULTI_CLAIM * gridDim.x * CWARPS < A.npairs)
                    ? MULTI_CLAIM
                    : 1u;
            u32 p0 = 0;
            if (lane == 0) p0 = atomicAdd(A.pair_counter, claim);
            p0 = __shfl_sync(FULL, p0, 0);
            pc = p0;
            pc_end = (p0 < A.npairs) ? min(A.npairs, p0 + claim) : p0;
          }
          p = pc++;
        } else {
          if (lane == 0) p = atomicAdd(A.pair_counter, 1u);
          p = __shfl_sync(FULL, p, 0);
        }
        if (p >= A.npairs) {
          exhausted = true;
          break;
        }
        // Step 2 (cu:198-235): sieve words for this pair
        const u32* P = A.pairs + 8ull * p;
        const u32 pw = (lane < 8) ? P[lane] : 0u;
        const u32 b0 = __shfl_sync(FULL, pw, 0), b1 = __shfl_sync(FULL, pw, 1);
        const u32 b2 = __shfl_sync(FULL, pw, 2), b3 = __shfl_sync(FULL, pw, 3);
        const u32 m0 = __shfl_sync(FULL, pw, 4);
        const u32 pline = MULTI ? (b3 >> 8) : 0u;
        ReqRec* prec = A.rec + pline;
        // thresholds: refreshed once per pair
        u32 t[4];
        {
          ull sk = 0, ek = 0;
          if (lane == 0) {
            sk = *(volatile ull*)&prec->st_key;
            ek = *(volatile ull*)&prec->e_key;
          }
          sk = __shfl_sync(FULL, sk, 0);
          ek = __shfl_sync(FULL, ek, 0);
          thr_st = (u32)sk;
          key_decode<4>(ek, t);
          if (!MULTI && lane < 4) W.thr[lane] = t[lane];
          thr3 = t[3];
          thr2 = t[2];
        }
        u32 bi = (A.bigindex >= 0) ? (u32)A.bigindex : (MULTI ? (b3 & 0xFFu) : b3);
        u32 f = A.tpo + bi;
        if (f >= POW3_COUNT) f = POW3_COUNT - 1;
        const u32 red = ((b0 % 9u) + 4u * (b1 % 9u) + 7u * (b2 % 9u)) % 9u;  // 2^32 = 4, 2^64 = 7 (mod 9)
        u32 word = A.mod9[red * 32u + lane];
        if (bi < 16u) {
          const u32 idx = (A.magic[bi] * m0) & ((1u << 24) - 1);
          const u32* row = A.bv + (size_t)bi * BV_WORDS + (idx >> 5);
          const u32 lo = row[lane];
          u32 hi = __shfl_down_sync(FULL, lo, 1);
          if (lane == 31) hi = row[32];
          word &= __funnelshift_r(lo, hi, idx & 31u);
        }
        u32 total;
        const u32 excl = warp_excl_scan(__popc(word), &total);
        if (total) {
          const u32 slot = ring_seq & (CR - 1);
          ring_seq++;
          const u32 rv = __shfl_sync(FULL, pw, lane < 3 ? lane : lane + 1);  // base0..2, number0..3
          if (lane < 7) W.ring[slot][lane] = rv;
          if (lane >= 7 && lane < 11) W.ring[slot][lane] = A.pow3[4u * f + (lane - 7)];
          if (lane == 11) W.ring[slot][11] = ((bi >= 16u) ? 1u : 0u) | (pline << 1);
          if (MULTI) {
            if (lane == 12) W.ring[slot][12] = thr_st;
            if (lane >= 13 && lane < 17) W.ring[slot][lane] = t[lane - 13];
            if (pline != wline) {  // seeds are counted per warp until the line changes
              if (lane == 0 && warp_seeds) atomicAdd(&A.rec[wline].seeds, warp_seeds);
              warp_seeds = 0;
              wline = pline;
            }
          }
          u32 pos = qhead + qcount + excl;
          while (word) {
            const u32 j = ctz32(word);
            word &= word - 1;
            W.q[pos & (CQ - 1)] = (unsigned short)((slot << 10) | (lane * 32u + j));
            pos++;
          }
          qcount += total;
          warp_seeds += total;
        }
        __syncwarp();
      }
      const u32 take = min(nidle, qcount);
      if (!active) {
        const u32 rank = __popc(idle & lanemask_lt());
        if (rank < take) {
          const u32 e = W.q[(qhead + rank) & (CQ - 1)];
          const u32* R = W.ring[e >> 10];
          const u32 a = e & 1023u;
          // seed n = base | a << (N-A)  (cu:241-260)
          n0 = R[0];
          n1 = R[1];
          n2 = R[2];
          {
            const u32 li = mbi >> 5, sh = mbi & 31u;
            const u32 lo = a << sh, hi = sh ? (a >> (32u - sh)) : 0u;
            if (li == 0) {
              n0 |= lo;
              n1 |= hi;
            } else if (li == 1) {
              n1 |= lo;
              n2 |= hi;
            } else {
              n2 |= lo;
            }
          }
          // v = number + a * 3^f  (cu:262-278)
          u64 t = (u64)a * R[7] + R[3];
          v0 = (u32)t;
          t = (u64)a * R[8] + R[4] + (t >> 32);
          v1 = (u32)t;
          t = (u64)a * R[9] + R[5] + (t >> 32);
          v2 = (u32)t;
          v3 = a * R[10] + R[6] + (u32)(t >> 32);
          cpu = R[11] & 1u;
          if (MULTI) {
            const u32 line = R[11] >> 1;
            if (line != hline) {  // this lane's XORs so far belong to the previous line
              if (hash) atomicXor(&A.rec[hline].hash, hash);
              hash = 0;
              hline = line;
            }
            W.lane[lane][8] = R[12];
            W.lane[lane][9] = R[13];
            W.lane[lane][10] = R[14];
            W.lane[lane][11] = R[15];
            W.lane[lane][12] = R[16];
            lthr_top = ((u64)R[16] << 32) | R[15];
          }
          nbl = bitlen96(n0, n1, n2);
          st = mbi;
          iters = 0;
          found = 0;
          ovf = 0;
          evalid = 0;
          if (n2 == 0 && n1 == 0 && n0 < 3u) {
            // v < n can never hold: the reference would loop forever
            atomicOr(&(MULTI ? A.rec + hline : A.rec)->errors, ERR_SEED_SMALL);
          } else {
            active = true;
            // E candidate T^(N-A)(n) = v - 1; (v3:v2) below the threshold's top limbs rejects it at once
            if ((((u64)v3 << 32) | v2) >= (MULTI ? lthr_top : (((u64)thr3 << 32) | thr2))) {
              const u32 x0 = v0 - 1, x1 = v1 - (v0 == 0), x2 = v2 - ((v0 | v1) == 0),
                        x3 = v3 - ((v0 | v1 | v2) == 0);
              const u32* th = MULTI ? &W.lane[lane][9] : W.thr;
              const bool ge = !lt96(x1, x2, x3, th[1], th[2], th[3]) &&
                              !((x3 == th[3]) & (x2 == th[2]) & (x1 == th[1]) & (x0 < th[0]));
              if (ge) {
                W.lane[lane][4] = x0;
                W.lane[lane][5] = x1;
                W.lane[lane][6] = x2;
                W.lane[lane][7] = x3;
                evalid = 1;
              }
            }
          }
        }
      }
      qhead = (qhead + take) & (CQ - 1);
      qcount -= take;
      if (take == 0 && exhausted && nidle == 32u) break;
    }

    // ---- Step 3 (cu:280-405) ----
    if (active) {
      const u64 thr_top = MULTI ? lthr_top : (((u64)thr3 << 32) | thr2);
      // one compare per odd run finds both rare events: v >= 2^100 (overflow, top limbs
      // 16:0) and, while the seed still counts, an excursion candidate (top limbs >= thr_top)
      constexpr u64 OVF_TOP = 16ull << 32;
      u64 gate = (found | ovf) ? OVF_TOP : min(thr_top, OVF_TOP);
#pragma unroll
      for (int it = 0; it < ITERS; it++) {
#pragma unroll
        for (int half = 0; half < 2; half++) {
          // 64-bit body while every lane of the group is below 2^59: an odd run of at most 8
          // steps multiplies by less than 2^5, so the value stays below 2^64 (the choice is
          // the same for all lanes that run this step together; lanes done have left the loop)
          const bool narrow = N64 && __all_sync(__activemask(), ((v2 | v3) == 0) & (v1 < (1u << 27)));
          if (N64 && narrow) {
            u64 v = ((u64)v1 << 32) | v0;
            const u32 a = ctz32(v0 | (1u << 8));
            v = (v >> a) * s_p3[a];
            st += a;
            v0 = (u32)v;
            v1 = (u32)(v >> 32);
            // (v3:v2) = 0 reaches the gate only when it is 0: no overflow, and the threshold
            // is below 2^64 while the seed still counts -- an excursion candidate
            if (gate == 0) CASES_EXC_CANDIDATE();
            const u64 x = v - 1;
            const u32 b = ctz32((u32)x | 0x80000000u);
            const u64 w = x >> b;
            if (!(found | ovf) & (b != 0) & ((n2 != 0) | (w < (((u64)n1 << 32) | n0)))) {
              sig = st + first_below((u32)x, (u32)(x >> 32), 0u, 0u, n0, n1, n2, nbl);
              found = 1;
              gate = OVF_TOP;
            }
            st += b;
            const u64 y = w + 1;
            v0 = (u32)y;
            v1 = (u32)(y >> 32);
          } else {
            // odd run; 3^a from registers.  The stopping time stops counting at the
            // first descent (found) or after an overflow report (ovf: no maxima).
            const u32 a = ctz32(v0 | (1u << 8));
            odd_run4(v0, v1, v2, v3, a, pow3_le8(a));
            st += a;
            if ((((u64)v3 << 32) | v2) >= gate) {  // overflow or excursion candidate (rare)
              if (v3 >= 16u) {  // v >= 2^100 (cu:295, 334); search3 tests > on the second (cu:702)
                const bool o = !(half == 1 && cpu && v3 == 16u && (v0 | v1 | v2) == 0u);
                if (o) {
                  const ull i = atomicAdd(A.overflow_count, 1ull);
                  if (i < A.overflow_cap) {
                    A.overflow[4 * i + 0] = n0;
                    A.overflow[4 * i + 1] = n1;
                    A.overflow[4 * i + 2] = n2;
                    A.overflow[4 * i + 3] = MULTI ? hline : 0u;
                  }
                  if (MULTI) atomicAdd(&A.rec[hline].items_done, 1ull);  // the line's overflow reports
                  ovf = 1;
                  gate = OVF_TOP;
                  v0 = 2;
                  v1 = v2 = v3 = 0;
                }
              }
              if (!found && !ovf && (((u64)v3 << 32) | v2) >= thr_top) CASES_EXC_CANDIDATE();
            }
            // even run
            v0 -= 1;
            const u32 b = ctz32(v0 | 0x80000000u);
            const u32 w0 = __funnelshift_r(v0, v1, b), w1 = __funnelshift_r(v1, v2, b);
            const u32 w2 = __funnelshift_r(v2, v3, b), w3 = v3 >> b;
            if (!(found | ovf) & (b != 0) & (w3 == 0) & lt96c(w0, w1, w2, n0, n1, n2)) {
              // first descent inside this run: smallest i with (v-1) >> i < n
              sig = st + first_below(v0, v1, v2, v3, n0, n1, n2, nbl);
              found = 1;
              gate = OVF_TOP;
            }
            st += b;
            v0 = w0 + 1;
            v1 = w1;
            v2 = w2;
            v3 = w3;
            add_carry3(v1, v2, v3, (v0 == 0) & (b != 0));  // carry of the +1 (cu:310-318)
          }
        }
        hash ^= v0;  // cu:359
        iters++;
        const bool done = (v3 == 0) & lt96c(v0, v1, v2, n0, n1, n2);  // cu:362-365
        if (done || iters >= A.iter_cap) {
          if (!done) {
            ReqRec* rec = MULTI ? A.rec + hline : A.rec;
            atomicOr(&rec->errors, ERR_ITER_CAP);
            atomicAdd(&rec->failures, 1ull);
          } else if (!ovf) {
            const u32 sigma = found ? sig : st;  // done implies found: an odd run only rises
            if (sigma >= (MULTI ? W.lane[lane][8] : thr_st)) {
              W.lane[lane][0] = sigma;
              pend |= 1u;
            }
            if (evalid) pend |= 2u;
            if (pend) {  // the seed, for the offer
              W.lane[lane][1] = n0;
              W.lane[lane][2] = n1;
              W.lane[lane][3] = n2;
              if (MULTI) W.lane[lane][MULTI ? 13 : 0] = hline;
            }
          }
          active = false;
          break;
        }
      }
    }
  }

  // ---- warp totals ----
  if (MULTI) {
    if (hash) atomicXor(&A.rec[hline].hash, hash);
    if (lane == 0 && warp_seeds) atomicAdd(&A.rec[wline].seeds, warp_seeds);
  } else {
#pragma unroll
    for (u32 d = 16; d; d >>= 1) hash ^= __shfl_xor_sync(FULL, hash, d);
    if (lane == 0) {
      atomicXor(&A.rec->hash, hash);
      atomicAdd(&A.rec->seeds, warp_seeds);
    }
  }
}

#undef CASES_EXC_CANDIDATE

// ------------------------------------------------------------------
// Host launcher.
// ------------------------------------------------------------------

template <int I, int R, bool N64 = false>
static cudaError_t launch_cases_t(const CasesArgs& a, u32 grid, cudaStream_t st) {
  if (a.multi) k_cases<I, R, true, N64><<<grid, CWARPS * 32, 0, st>>>(a);
  else k_cases<I, R, false, N64><<<grid, CWARPS * 32, 0, st>>>(a);
  return cudaGetLastError();
}

// Variants: checkpoints per pass and refill threshold; variant 4 adds the 64-bit body
// (for N <= 52; variant 3 above).
int cases_variants() { return 5; }

cudaError_t launch_cases(const CasesArgs& a, int variant, u32 grid, cudaStream_t st) {
  // seeds n = base | a << (N - A) lie below 2^N (A = 10): above 2^52 the 128-bit body alone is faster
  if (variant == 4 && a.mbi + 10u > RANGE_NARROW_MAX_BITS) variant = 3;
  switch (variant) {
    case 0: return launch_cases_t<1, 1>(a, grid, st);
    case 1: return launch_cases_t<2, 4>(a, grid, st);
    case 2: return launch_cases_t<2, 8>(a, grid, st);
    case 4: return launch_cases_t<4, 8, true>(a, grid, st);
    default: return launch_cases_t<4, 8>(a, grid, st);
  }
}

template <bool M>
static cudaError_t occupancy_t(int variant, int* bps) {
  switch (variant) {
    case 0: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_cases<1, 1, M>, CWARPS * 32, 0);
    case 1: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_cases<2, 4, M>, CWARPS * 32, 0);
    case 2: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_cases<2, 8, M>, CWARPS * 32, 0);
    case 4: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_cases<4, 8, M, true>, CWARPS * 32, 0);
    default: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_cases<4, 8, M>, CWARPS * 32, 0);
  }
}

cudaError_t cases_occupancy(int variant, int* blocks_per_sm, bool multi) {
  return multi ? occupancy_t<true>(variant, blocks_per_sm) : occupancy_t<false>(variant, blocks_per_sm);
}

}  // namespace cz
