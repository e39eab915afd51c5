// range_shared.cuh -- pieces shared by the range kernels (range.cu: the
// general kernel with four-limb values; range64.cu: the kernel with 64-bit
// values): constants of the work distribution and the mod-9 sieve, the
// staged work item and its cp.async staging from the survivor table, and
// the widening hand-off.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"
#include "tables.h"

namespace cz {

constexpr u32 RQ = 128;          // queue entries per warp, power of two (>= 32 R + one item)
constexpr u32 RR = 32;           // item slots per warp (one per lane; see the expansions)
constexpr u32 CLAIM = 8;         // items claimed per atomic near the end of a launch
constexpr u32 CLAIM_BIG = 32;    // ... and while at least 128 items per warp remain
constexpr u32 KEEP9 = 0xCBu;     // n mod 9 in {0,1,3,6,7} survives (cu:488)
// Negative variant T'(m) = (3m-1)/2, m/2: m = 1 mod 3 (m > 1) is T' of the smaller
// (2m+1)/3 and m = 5 mod 9 (m > 5) is T'^3 of the smaller (8m+5)/9, so m mod 9 in
// {0,2,3,6,8} survives (and m = 5, the minimum of a cycle).
constexpr u32 KEEP9N = 0x14Du;
constexpr u32 OVF3 = 1u << 23;   // v >= 2^119 after an odd run: the next run could leave 128 bits
constexpr u32 ST_CAP = 1u << 20; // steps per seed before ERR_ITER_CAP

// The work item staged for expansion (warp-uniform).
struct StagedItem {
  ull q_lo;      // kind 0: block q (low 64 bits); kind 1: first integer
  ull d_hi;      // kind 1: end (exclusive)
  u32 q_hi;      // kind 0: block q bits 64..95
  u32 sbase, send;  // kind 0: survivor-table range of the item
  u32 req, kind, mod9, valid, pad;
};

__device__ __forceinline__ u32 mod9_96(u32 a0, u32 a1, u32 a2) {
  return ((a0 % 9u) + 4u * (a1 % 9u) + 7u * (a2 % 9u)) % 9u;
}

// Bits 32..95 of a value below 2^128 given as limbs 1..3; all ones when it
// is >= 2^96.  Comparing this window is a conservative excursion test.
__device__ __forceinline__ u64 gate_window(u32 x1, u32 x2, u32 x3) {
  return x3 ? ~0ull : (((u64)x2 << 32) | x1);
}

__device__ __forceinline__ u32 bitlen128(unsigned __int128 x) {
  const u64 hi = (u64)(x >> 64), lo = (u64)x;
  return hi ? 128u - __clzll(hi) : (lo ? 64u - __clzll(lo) : 0u);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The trajectory value a run state stands for: T^s(n) = v - 1 (the state is
// v = T^s(n) + 1), or for the negative variant T'^s(n) = u + 1 (the state is
// u = T'^s(n) - 1).
template <bool NEG>
__device__ __forceinline__ void value_of(u32 v0, u32 v1, u32 v2, u32 v3, u32* x) {
  if (NEG) {
    x[0] = v0 + 1;
    const u32 c0 = x[0] == 0;
    x[1] = v1 + c0;
    const u32 c1 = c0 & (x[1] == 0);
    x[2] = v2 + c1;
    x[3] = v3 + (c1 & (x[2] == 0));
  } else {
    x[0] = v0 - 1;
    x[1] = v1 - (v0 == 0);
    x[2] = v2 - ((v0 | v1) == 0);
    x[3] = v3 - ((v0 | v1 | v2) == 0);
  }
}

// Queue a seed for the 192/256-bit re-run.
__device__ __forceinline__ void widen_seed(const RangeArgs& A, u32 req, u32 n0, u32 n1, u32 n2) {
  const u32 wi = atomicAdd(A.widen_count, 1u);
  if (wi < A.widen_cap) {
    A.widen[wi] = WidenEntry{req, n0, n1, n2};
    atomicAdd(&A.recs[req].widened, 1ull);
  } else {
    atomicOr(&A.recs[req].errors, ERR_WIDEN_FULL);
    atomicAdd(&A.recs[req].failures, 1ull);
  }
}

// Advances to the next work item (claiming CLAIM items at a time), resolves
// its segment and block, and starts copying its survivor entries into dst
// with cp.async so that they arrive while the current item is worked on.
// Warp-uniform; lane 0 owns the bookkeeping.  WT is the kernel's per-warp
// state (fields seg, nxt, item, claim_hi, seg_lo, seg_hi, qi, chunk).
template <class WT>
__device__ __forceinline__ void stage_next(WT& W, uint4* dst, const RangeArgs& A, const uint4* __restrict__ T,
                                           u32 lane) {
  ull next = W.item + 1;
  bool fresh = false;
  if (next >= W.claim_hi) {
    // the warp's last claim end stands in for the cursor: big claims while far from the end
    const u32 claim =
        (W.claim_hi + (ull)gridDim.x * (blockDim.x >> 5) * 128u < A.item_limit) ? CLAIM_BIG : CLAIM;
    ull c = 0;
    if (lane == 0) c = atomicAdd(A.item_cursor, (ull)claim);
    c = __shfl_sync(FULL, c, 0);
    if (c >= A.item_limit) {
      __syncwarp();
      if (lane == 0) W.nxt.valid = 0;
      __syncwarp();
      return;
    }
    next = c;
    fresh = true;
    __syncwarp();
    if (lane == 0) W.claim_hi = min(c + claim, A.item_limit);
  }
  if (next < W.seg_lo || next >= W.seg_hi) {
    u32 si = 0;
    if (lane == 0) {
      u32 lo = 0, hi = A.nsegs;
      while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (A.segs[mid].item_begin <= next) lo = mid; else hi = mid;
      }
      si = lo;
    }
    si = __shfl_sync(FULL, si, 0);
    __syncwarp();
    const u32* src = reinterpret_cast<const u32*>(A.segs + si);
    if (lane < sizeof(RangeSeg) / 4) reinterpret_cast<u32*>(&W.seg)[lane] = src[lane];
    if (lane == 0) {
      W.seg_lo = A.segs[si].item_begin;
      W.seg_hi = (si + 1 < A.nsegs) ? A.segs[si + 1].item_begin : A.item_limit;
    }
    fresh = true;
    __syncwarp();
  }
  ull qi;
  u32 chunk;
  const u32 kind = W.seg.kind;
  if (fresh) {
    const ull local = next - W.seg_lo + (((ull)W.seg.local0_hi << 32) | W.seg.local0_lo);
    if (kind == 0) {  // segments hold fewer than 2^32 items
      const u32 l32 = (u32)local, ipq = W.seg.ipq;
      const u32 q32 = l32 / ipq;
      qi = q32;
      chunk = l32 - q32 * ipq;
    } else {
      qi = local;
      chunk = 0;
    }
  } else if (kind == 0) {
    qi = W.qi;
    chunk = W.chunk + 1;
    if (chunk == W.seg.ipq) {
      chunk = 0;
      qi++;
    }
  } else {
    qi = W.qi + 1;
    chunk = 0;
  }
  StagedItem it;
  it.req = W.seg.req;
  it.kind = kind;
  it.mod9 = W.seg.mod9;
  it.valid = 1;
  it.pad = 0;
  if (kind == 0) {
    const u32 qs = W.seg.qstride ? W.seg.qstride : 1u;
    const unsigned __int128 q = (((unsigned __int128)W.seg.q_hi << 64) | W.seg.q_lo) + (unsigned __int128)qi * qs;
    it.q_lo = (u64)q;
    it.q_hi = (u32)(q >> 64);
    it.sbase = W.seg.s_lo + chunk * RANGE_ITEM;
    it.send = min(it.sbase + RANGE_ITEM, W.seg.s_hi);
    it.d_hi = 0;
#pragma unroll
    for (u32 j = 0; j < RANGE_ITEM / 32; j++) {
      const u32 idx = it.sbase + j * 32 + lane;
      if (idx < it.send) cp_async16(&dst[j * 32 + lane], T + idx);
    }
    cp_async_commit();
  } else {
    it.q_lo = W.seg.q_lo + qi * DENSE_ITEM;
    it.q_hi = 0;
    it.sbase = it.send = 0;
    it.d_hi = W.seg.d_hi;
  }
  __syncwarp();
  if (lane == 0) {
    W.item = next;
    W.qi = qi;
    W.chunk = chunk;
    W.nxt = it;
  }
  __syncwarp();
}

// Table of J steps for residues r < 2^J (J <= 11): T^J(r) [17:0] | f_J [21:18]
// | bitlen(g) [26:22] | bitlen(h) [31:27], g and h the least and largest of
// 2^(J-i) 3^(f_i) over 1 <= i <= J.  For x = a 2^J + r, T^i(x) = a 2^(J-i) 3^(f_i)
// + T^i(r) with 0 <= T^i(r) < 2^(J-i) 3^(f_i), so a g <= T^i(x) < (a + 1) h.
__device__ __forceinline__ void build_step_table(u32* t, u32 J) {
  for (u32 r = threadIdx.x; r < (1u << J); r += blockDim.x) {
    u32 x = r, f = 0, g = 0xFFFFFFFFu, h = 0;
    for (u32 i = 1; i <= J; i++) {
      if (x & 1u) {
        x = x + (x >> 1) + 1u;  // (3x + 1) / 2
        f++;
      } else {
        x >>= 1;
      }
      u32 m = 1u << (J - i);
      for (u32 j = 0; j < f; j++) m *= 3u;
      g = min(g, m);
      h = max(h, m);
    }
    t[r] = x | (f << 18) | ((32u - __clz(g)) << 22) | ((32u - __clz(h)) << 27);
  }
}

}  // namespace cz
