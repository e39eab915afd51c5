// range.cu -- range verification: every seed n of [offset, offset+size)
// that survives the 2^k residue sieve and the mod-9 sieve is iterated
// until it falls below its start; outputs are the seeds checked, the
// maximum stopping time and the maximum excursion (each with the smallest
// seed on ties) and the seeds that did not finish.
//
// One kernel serves the plain single range and the batched form: the
// host lowers every request into segments of work items, and persistent
// warps claim items from a global cursor.  A sieved item is 256 consecutive
// entries of the survivor table for one block q (seeds n = q 2^k + r); the
// warp reads them with coalesced 16-byte loads, applies the mod-9 sieve
// (n mod 9 from q mod 9 and the stored r mod 9), ranks the survivors with
// popc + a warp scan into its shared-memory queue, and idle lanes pull
// seeds from the queue.  A seed starts after one k-step jump,
// T^k(n) + 1 = q 3^f + c (no descent is possible in those k steps), then
// runs odd/even runs in 4 x 32-bit limbs with the exact stopping time and
// excursion.  A value that could leave 2^128 sends the seed to the widen
// list, re-run from scratch with 6 and then 8 limbs.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"
#include "tables.h"

namespace cz {

constexpr u32 RQ = 1024;  // queue entries per warp (>= 31 + survivors of one dense item)
constexpr u32 RR = 32;    // item slots per warp
constexpr u32 RWARPS = 8;
constexpr u32 KEEP9 = 0xCBu;  // n mod 9 in {0,1,3,6,7} survives (cu:488)

struct RangeWarp {
  unsigned short q[RQ];  // (slot << 10) | local index
  u32 ring[RR][12];      // [0] kind [1] s_base [2..4] q / d limbs [5] req [6] thr_st [7] thr bit length [8..11] thrE
  u32 lane[32][12];      // [0] st [1..3] seed [4..7] seed-local max E [8..11] thrE
};

__device__ __forceinline__ u32 mod9_96(u32 a0, u32 a1, u32 a2) {
  return ((a0 % 9u) + 4u * (a1 % 9u) + 7u * (a2 % 9u)) % 9u;
}

// x >= ref for 4-limb values
__device__ __forceinline__ bool ge128(u32 x0, u32 x1, u32 x2, u32 x3, const u32* ref) {
  return !(lt96(x1, x2, x3, ref[1], ref[2], ref[3]) ||
           ((x3 == ref[3]) & (x2 == ref[2]) & (x1 == ref[1]) & (x0 < ref[0])));
}

template <int ITERS, int REFILL_MIN>
__global__ void __launch_bounds__(RWARPS * 32) k_range(const RangeArgs A) {
  __shared__ RangeWarp S[RWARPS];
  __shared__ unsigned long long s_p3[41];
  __shared__ u32 s_pow3[9], s_keep9[9];
  const u32 lane = lane_id();
  RangeWarp& W = S[threadIdx.x >> 5];
  if (threadIdx.x < 41) {
    unsigned long long p = 1;
    for (u32 i = 0; i < threadIdx.x; i++) p *= 3;
    s_p3[threadIdx.x] = p;
    if (threadIdx.x < 9) s_pow3[threadIdx.x] = (u32)p;
  }
  if (threadIdx.x >= 64 && threadIdx.x < 73) {
    const u32 r = threadIdx.x - 64;  // bit j: (r + j) mod 9 survives
    u32 m = 0;
    for (u32 j = 0; j < 32; j++) m |= ((KEEP9 >> ((r + j) % 9u)) & 1u) << j;
    s_keep9[r] = m;
  }
  __syncthreads();

  const u32 k = A.k;
  const u32 k9 = (u32)((1ull << (k % 6)) % 9ull);  // 2^k mod 9 (2^6 = 1 mod 9)
  // warp-uniform state
  u32 qhead = 0, qcount = 0, ring_seq = 0;
  bool exhausted = false;
  // lane state
  bool active = false;
  u32 v0 = 0, v1 = 0, v2 = 0, v3 = 0, n0 = 0, n1 = 0, n2 = 0;
  u32 st = 0, iters = 0, evalid = 0, pend = 0, req = 0, thr_st = 0;
  u64 thr_top = 0;

  for (;;) {
    // ---- offers of finished seeds, one lane at a time ----
    {
      u32 pm = __ballot_sync(FULL, pend != 0);
      while (pm) {
        const u32 leader = __ffs(pm) - 1;
        if (lane == leader) {
          const u32 seed[4] = {W.lane[lane][1], W.lane[lane][2], W.lane[lane][3], 0};
          if (pend & 1u) rec_offer_st(A.recs + req, W.lane[lane][0], seed);
          if (pend & 2u) rec_offer_e<4>(A.recs + req, &W.lane[lane][4], seed);
          pend = 0;
        }
        pm &= pm - 1;
      }
      __syncwarp();
    }

    // ---- refill ----
    const u32 idle = __ballot_sync(FULL, !active);
    const u32 nidle = __popc(idle);
    if (nidle >= (u32)REFILL_MIN || nidle == 32u) {
      while (qcount < nidle && !exhausted) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(A.item_cursor, 1ull);
        item = __shfl_sync(FULL, item, 0);
        if (item >= A.item_limit) {
          exhausted = true;
          break;
        }
        // segment of this item (binary search; the last segment with item_begin <= item)
        u32 si = 0;
        if (lane == 0) {
          u32 lo = 0, hi = A.nsegs;
          while (hi - lo > 1) {
            const u32 mid = (lo + hi) >> 1;
            if (A.segs[mid].item_begin <= item) lo = mid; else hi = mid;
          }
          si = lo;
        }
        si = __shfl_sync(FULL, si, 0);
        const RangeSeg& G = A.segs[si];
        const unsigned long long local = item - G.item_begin;
        const u32 rq = G.req;
        ReqRec* R = A.recs + rq;
        ull sk = 0, ek = 0;
        if (lane == 0) {
          sk = *(volatile ull*)&R->st_key;
          ek = *(volatile ull*)&R->e_key;
        }
        sk = __shfl_sync(FULL, sk, 0);
        ek = __shfl_sync(FULL, ek, 0);
        u32 mask = 0, kind = G.kind, sbase = 0, q0 = 0, q1 = 0, q2 = 0;
        if (kind == 0) {
          const unsigned long long qi = local / G.ipq;
          const u32 chunk = (u32)(local - qi * G.ipq);
          const unsigned __int128 q = (((unsigned __int128)G.q_hi << 64) | G.q_lo) + qi;
          q0 = (u32)q;
          q1 = (u32)(q >> 32);
          q2 = (u32)(q >> 64);
          sbase = G.s_lo + chunk * RANGE_ITEM;
          const u32 send = min(sbase + RANGE_ITEM, G.s_hi);
          const u32 b9 = (mod9_96(q0, q1, q2) * k9) % 9u;
          const uint4* T = reinterpret_cast<const uint4*>(A.table);
#pragma unroll
          for (u32 j = 0; j < RANGE_ITEM / 32; j++) {
            const u32 idx = sbase + j * 32 + lane;
            if (idx < send) {
              const uint4 e = T[idx];
              u32 x = b9 + ((e.y >> 16) & 0xFFu);
              x = (x >= 9u) ? x - 9u : x;
              if (!G.mod9 || ((KEEP9 >> x) & 1u)) mask |= 1u << j;
            }
          }
        } else {
          const unsigned long long d = G.q_lo + local * DENSE_ITEM + 32ull * lane;
          q0 = (u32)(G.q_lo + local * DENSE_ITEM);
          q1 = (u32)((G.q_lo + local * DENSE_ITEM) >> 32);
          if (d < G.d_hi) {
            const unsigned long long cnt = G.d_hi - d;
            mask = (cnt >= 32) ? FULL : ((1u << cnt) - 1u);
            if (G.mod9) mask &= s_keep9[d % 9u];
            if (d < 2) mask &= ~((d == 0) ? 3u : 1u);  // n = 0, 1 have no stopping time
          }
        }
        u32 total;
        const u32 excl = warp_excl_scan(__popc(mask), &total);
        if (lane == 0) {
          if (total) atomicAdd(&R->seeds, (ull)total);
          atomicAdd(&R->items_done, 1ull);
        }
        if (total) {
          const u32 slot = ring_seq & (RR - 1);
          ring_seq++;
          u32 t[4];
          key_decode<4>(ek, t);
          const u32 thr_bl = (u32)(ek >> 54);
          u32 rv = 0;
          switch (lane) {
            case 0: rv = kind; break;
            case 1: rv = sbase; break;
            case 2: rv = q0; break;
            case 3: rv = q1; break;
            case 4: rv = q2; break;
            case 5: rv = rq; break;
            case 6: rv = (u32)min(sk, 0xFFFFFFFFull); break;
            case 7: rv = thr_bl; break;
            case 8: rv = t[0]; break;
            case 9: rv = t[1]; break;
            case 10: rv = t[2]; break;
            case 11: rv = t[3]; break;
          }
          if (lane < 12) W.ring[slot][lane] = rv;
          u32 pos = qhead + qcount + excl;
          const u32 mm = mask;
          u32 m = mm;
          while (m) {
            const u32 j = ctz32(m);
            m &= m - 1;
            const u32 li = (kind == 0) ? (j * 32u + lane) : (lane * 32u + j);
            W.q[pos & (RQ - 1)] = (unsigned short)((slot << 10) | li);
            pos++;
          }
          qcount += total;
        }
        __syncwarp();
      }
      const u32 take = min(nidle, qcount);
      if (!active) {
        const u32 rank = __popc(idle & lanemask_lt());
        if (rank < take) {
          const u32 e = W.q[(qhead + rank) & (RQ - 1)];
          const u32* G = W.ring[e >> 10];
          const u32 li = e & 1023u;
          req = G[5];
          thr_st = G[6];
          const u32 thr_bl = G[7];
          W.lane[lane][8] = G[8];
          W.lane[lane][9] = G[9];
          W.lane[lane][10] = G[10];
          W.lane[lane][11] = G[11];
          thr_top = ((u64)G[11] << 32) | G[10];
          unsigned __int128 N, V;
          bool replay = true;
          if (G[0] == 0) {
            const uint4 en = reinterpret_cast<const uint4*>(A.table)[G[1] + li];
            const unsigned __int128 Q = ((unsigned __int128)G[4] << 64) | ((u64)G[3] << 32) | G[2];
            const u64 r = (u64)en.x | ((u64)(en.y & 0xFFu) << 32);
            const u32 f = (en.y >> 8) & 0xFFu, emax = en.y >> 24;
            N = (Q << k) | r;
            const u32 nbl = (u32)(N >> 64) ? 128u - __clzll((u64)(N >> 64)) : 64u - __clzll((u64)N);
            // all of T^0..T^k(n) < 2^emax (n + 1 + k) <= 2^(bitlen(n) + 1 + emax) <= threshold: skip them
            replay = nbl + 1 + emax >= thr_bl;
            if (!replay) {
              V = Q * (unsigned __int128)s_p3[f] + (((u64)en.w << 32) | en.z);
              st = k;
            }
          } else {
            N = ((u64)G[3] << 32 | G[2]) + (u64)li;
          }
          if (replay) {
            V = N + 1;
            st = 0;
          }
          n0 = (u32)N;
          n1 = (u32)(N >> 32);
          n2 = (u32)(N >> 64);
          v0 = (u32)V;
          v1 = (u32)(V >> 32);
          v2 = (u32)(V >> 64);
          v3 = (u32)(V >> 96);
          iters = 0;
          evalid = 0;
          active = true;
          // excursion candidate: n itself, or T^k(n) = v - 1 after the jump
          const unsigned __int128 X = V - 1;
          const u32 x0 = (u32)X, x1 = (u32)(X >> 32), x2 = (u32)(X >> 64), x3 = (u32)(X >> 96);
          if (ge128(x0, x1, x2, x3, &W.lane[lane][8])) {
            W.lane[lane][4] = x0;
            W.lane[lane][5] = x1;
            W.lane[lane][6] = x2;
            W.lane[lane][7] = x3;
            evalid = 1;
          }
        }
      }
      qhead = (qhead + take) & (RQ - 1);
      qcount -= take;
      if (take == 0 && exhausted && nidle == 32u) break;
    }

    // ---- iterate ----
    if (active) {
#pragma unroll 1
      for (int it = 0; it < ITERS; it++) {
        bool done = false, widen = false;
        if (v3 >= (1u << 19)) {
          widen = true;  // (v >> a) 3^a could leave 128 bits
        } else {
          const u32 a = ctz32(v0 | (1u << 8));
          odd_run4(v0, v1, v2, v3, a, s_pow3[a]);
          st += a;
          if ((((u64)v3 << 32) | v2) >= thr_top) {
            const u32 x0 = v0 - 1, x1 = v1 - (v0 == 0), x2 = v2 - ((v0 | v1) == 0), x3 = v3 - ((v0 | v1 | v2) == 0);
            const u32* ref = evalid ? &W.lane[lane][4] : &W.lane[lane][8];
            if (ge128(x0, x1, x2, x3, ref)) {
              W.lane[lane][4] = x0;
              W.lane[lane][5] = x1;
              W.lane[lane][6] = x2;
              W.lane[lane][7] = x3;
              evalid = 1;
            }
          }
          v0 -= 1;
          const u32 b = ctz32(v0 | 0x80000000u);
          const u32 w0 = __funnelshift_r(v0, v1, b), w1 = __funnelshift_r(v1, v2, b);
          const u32 w2 = __funnelshift_r(v2, v3, b), w3 = v3 >> b;
          if (b != 0 && w3 == 0 && w2 <= n2 && lt96(w0, w1, w2, n0, n1, n2)) {
            u32 i = 1;
            for (; i < b; i++) {
              const u32 y0 = __funnelshift_r(v0, v1, i), y1 = __funnelshift_r(v1, v2, i);
              const u32 y2 = __funnelshift_r(v2, v3, i), y3 = v3 >> i;
              if (y3 == 0 && lt96(y0, y1, y2, n0, n1, n2)) break;
            }
            st += i;
            done = true;
          } else {
            st += b;
            v0 = w0 + 1;
            v1 = w1;
            v2 = w2;
            v3 = w3;
            if (v0 == 0 && b != 0) {
              v1 += 1;
              if (v1 == 0) {
                v2 += 1;
                if (v2 == 0) v3 += 1;
              }
            }
          }
        }
        if (done) {
          W.lane[lane][1] = n0;
          W.lane[lane][2] = n1;
          W.lane[lane][3] = n2;
          if (st >= thr_st) {
            W.lane[lane][0] = st;
            pend |= 1u;
          }
          if (evalid) pend |= 2u;
          active = false;
          break;
        }
        if (widen || ++iters >= A.iter_cap) {
          if (widen) {
            const u32 wi = atomicAdd(A.widen_count, 1u);
            if (wi < A.widen_cap) {
              A.widen[wi] = WidenEntry{req, n0, n1, n2};
              atomicAdd(&A.recs[req].widened, 1ull);
            } else {
              atomicOr(&A.recs[req].errors, ERR_WIDEN_FULL);
              atomicAdd(&A.recs[req].failures, 1ull);
            }
          } else {
            atomicOr(&A.recs[req].errors, ERR_ITER_CAP);
            atomicAdd(&A.recs[req].failures, 1ull);
          }
          active = false;
          break;
        }
      }
    }
  }
}

// ------------------------------------------------------------------
// Wide re-run: one seed per thread with L limbs, from scratch.
// ------------------------------------------------------------------
template <int L>
__global__ void __launch_bounds__(128) k_range_wide(const WidenEntry* __restrict__ list, const u32* count,
                                                   u32 cap, ReqRec* recs, WidenEntry* next, u32 next_cap,
                                                   u32* next_count, u32 iter_cap) {
  const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  const u32 n = min(*count, cap);
  const u32 lane = lane_id();
  bool ok = false;
  WidenEntry e{0, 0, 0, 0};
  Limbs<L> v, N, E;
  unsigned long long st = 0;
  if (i < n) {
    e = list[i];
#pragma unroll
    for (int j = 0; j < L; j++) N.w[j] = (j == 0) ? e.n0 : (j == 1) ? e.n1 : (j == 2) ? e.n2 : 0u;
    v = N;
    inc_l<L>(v);
    E = N;
    u32 it = 0;
    for (;;) {
      if (v.w[L - 1] >= (1u << 19) || ++it > iter_cap) {
        if (it > iter_cap) {
          atomicOr(&recs[e.req].errors, ERR_ITER_CAP);
          atomicAdd(&recs[e.req].failures, 1ull);
        } else if (next) {
          const u32 wi = atomicAdd(next_count, 1u);
          if (wi < next_cap) {
            next[wi] = e;
          } else {
            atomicOr(&recs[e.req].errors, ERR_WIDEN_FULL);
            atomicAdd(&recs[e.req].failures, 1ull);
          }
        } else {
          atomicAdd(&recs[e.req].failures, 1ull);
        }
        break;
      }
      const u32 a = ctz32(v.w[0] | (1u << 8));
      u32 m = 1;
      for (u32 j = 0; j < a; j++) m *= 3u;
      odd_run_l<L>(v, a, m);
      st += a;
      Limbs<L> x = v;
      dec_l<L>(x);
      if (limbs_lt<L>(E, x)) E = x;
      // even run on x = v - 1
      const u32 b = ctz32(x.w[0] | 0x80000000u);
      Limbs<L> w = x;
      shr_l<L>(w, b);
      if (b != 0 && limbs_lt<L>(w, N)) {
        u32 s = 1;
        for (; s < b; s++) {
          Limbs<L> y = x;
          shr_l<L>(y, s);
          if (limbs_lt<L>(y, N)) break;
        }
        st += s;
        ok = true;
        break;
      }
      st += b;
      v = w;
      inc_l<L>(v);
    }
  }
  u32 pm = __ballot_sync(FULL, ok);
  while (pm) {
    const u32 leader = __ffs(pm) - 1;
    if (lane == leader) {
      const u32 seed[4] = {e.n0, e.n1, e.n2, 0};
      rec_offer_st(recs + e.req, st, seed);
      rec_offer_e<L>(recs + e.req, E.w, seed);
    }
    pm &= pm - 1;
  }
}

// ------------------------------------------------------------------
// Launchers.
// ------------------------------------------------------------------
int range_variants() { return 4; }

#define CZ_RANGE_VARIANTS(X) X(0, 4, 1) X(1, 4, 4) X(2, 8, 4) X(3, 8, 8)

cudaError_t launch_range(const RangeArgs& a, int variant, u32 grid, cudaStream_t st) {
  switch (variant) {
#define X(id, it, rm) \
  case id:            \
    k_range<it, rm><<<grid, RWARPS * 32, 0, st>>>(a); break;
    CZ_RANGE_VARIANTS(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t range_occupancy(int variant, int* bps) {
  switch (variant) {
#define X(id, it, rm) \
  case id:            \
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_range<it, rm>, RWARPS * 32, 0);
    CZ_RANGE_VARIANTS(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_range_wide(const WidenEntry* list, const u32* count, u32 cap, int limbs, ReqRec* recs,
                              WidenEntry* next, u32 next_cap, u32* next_count, u32 iter_cap, cudaStream_t st) {
  const u32 grid = (cap + 127) / 128;
  if (limbs == 6)
    k_range_wide<6><<<grid, 128, 0, st>>>(list, count, cap, recs, next, next_cap, next_count, iter_cap);
  else
    k_range_wide<8><<<grid, 128, 0, st>>>(list, count, cap, recs, nullptr, 0, nullptr, iter_cap);
  return cudaGetLastError();
}

}  // namespace cz
