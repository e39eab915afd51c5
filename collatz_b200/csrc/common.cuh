// common.cuh -- device helpers shared by the sieve, cases, range and
// trajectory kernels: 32-bit-limb arithmetic for the run-length Collatz
// step, warp scans, the monotone excursion key, and bounded record locks.
//
// Values are kept in the reference's "+1" space, v = T^k(n) + 1 (main.rs:13,
// collatz_cudav7.cu:280-405): an odd run of length a is v -> 3^a (v >> a),
// an even run of length b is v -> ((v - 1) >> b) + 1.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rec.h"

namespace cz {

typedef uint32_t u32;
typedef uint64_t u64;
typedef unsigned long long ull;

constexpr u32 FULL = 0xFFFFFFFFu;
constexpr u32 BV_WORDS = (1u << 19) + 32u;  // one look-ahead bit vector, cu:68
constexpr u32 LOCK_SPIN_LIMIT = 1u << 20;   // bounded spin on record locks

__device__ __forceinline__ u32 lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ u32 lanemask_lt() {
  u32 m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Trailing zeros of a non-zero word.
__device__ __forceinline__ u32 ctz32(u32 x) { return (u32)(__ffs((int)x) - 1); }

// Warp-wide exclusive prefix sum; *total receives the sum over the warp.
__device__ __forceinline__ u32 warp_excl_scan(u32 x, u32* total) {
  const u32 lane = lane_id();
  u32 incl = x;
#pragma unroll
  for (u32 d = 1; d < 32; d <<= 1) {
    u32 y = __shfl_up_sync(FULL, incl, d);
    if (lane >= d) incl += y;
  }
  *total = __shfl_sync(FULL, incl, 31);
  return incl - x;
}

// (a2,a1,a0) < (b2,b1,b0), unsigned 96-bit.
__device__ __forceinline__ bool lt96(u32 a0, u32 a1, u32 a2, u32 b0, u32 b1, u32 b2) {
  return (a2 < b2) | ((a2 == b2) & ((a1 < b1) | ((a1 == b1) & (a0 < b0))));
}

// 3^a for a <= 7 from two byte-permute lookups: low bytes 01 03 09 1B 51 F3 D9 8B,
// high bytes 00 00 00 00 00 00 02 08 (3^6 = 0x2D9, 3^7 = 0x88B).
__device__ __forceinline__ u32 pow3_le7(u32 a) {
  return (__byte_perm(0x1B090301u, 0x8BD9F351u, a) & 0xFFu) | __byte_perm(0u, 0x08020000u, a << 4);
}

// 3^a for a <= 8 (3^8 = 6561), in registers.
__device__ __forceinline__ u32 pow3_le8(u32 a) { return a == 8u ? 6561u : pow3_le7(a); }

// (a2:a1:a0) < (b2:b1:b0) as one borrow chain.
__device__ __forceinline__ bool lt96c(u32 a0, u32 a1, u32 a2, u32 b0, u32 b1, u32 b2) {
  u32 r;
  asm("{\n\t.reg .u32 t;\n\t"
      "sub.cc.u32 t, %1, %4;\n\t"
      "subc.cc.u32 t, %2, %5;\n\t"
      "subc.cc.u32 t, %3, %6;\n\t"
      "subc.u32 %0, 0, 0;\n\t}"
      : "=r"(r)
      : "r"(a0), "r"(a1), "r"(a2), "r"(b0), "r"(b1), "r"(b2));
  return r != 0;
}

// (v3:v2:v1) += c for c in {0, 1}, as one carry chain.
__device__ __forceinline__ void add_carry3(u32& v1, u32& v2, u32& v3, u32 c) {
  asm("add.cc.u32 %0, %0, %3;\n\t"
      "addc.cc.u32 %1, %1, 0;\n\t"
      "addc.u32 %2, %2, 0;"
      : "+r"(v1), "+r"(v2), "+r"(v3)
      : "r"(c));
}

// Bit length of a 96-bit value.
__device__ __forceinline__ u32 bitlen96(u32 n0, u32 n1, u32 n2) {
  return n2 ? 96u - __clz(n2) : (n1 ? 64u - __clz(n1) : 32u - __clz(n0));
}

// Least i >= 1 with (x >> i) < n, for x = (x3:x2:x1:x0) and a 96-bit n of bit
// length bln, given that x >> b < n for some b <= 31.  With d = bitlen(x) -
// bln: x >> i has more bits than n for i < d, fewer for i = d + 1, so the
// answer is d or d + 1 (1 when d < 1).  Constant time, no loop over i.
__device__ __forceinline__ u32 first_below(u32 x0, u32 x1, u32 x2, u32 x3, u32 n0, u32 n1, u32 n2, u32 bln) {
  const u32 bx = x3 ? 128u - __clz(x3) : (x2 ? 96u - __clz(x2) : (x1 ? 64u - __clz(x1) : 32u - __clz(x0)));
  const int d = (int)bx - (int)bln;
  if (d < 1) return 1u;
  const u32 y0 = __funnelshift_r(x0, x1, d), y1 = __funnelshift_r(x1, x2, d);
  const u32 y2 = __funnelshift_r(x2, x3, d), y3 = x3 >> d;
  return ((y3 == 0) & lt96(y0, y1, y2, n0, n1, n2)) ? (u32)d : (u32)d + 1u;
}

// Odd run on 4 limbs: v <- (v >> a) * m with m = 3^a, a <= 8
// (collatz_cudav7.cu:282-293).  The product is taken mod 2^128.
__device__ __forceinline__ void odd_run4(u32& v0, u32& v1, u32& v2, u32& v3, u32 a, u32 m) {
  const u32 t0 = __funnelshift_r(v0, v1, a);
  const u32 t1 = __funnelshift_r(v1, v2, a);
  const u32 t2 = __funnelshift_r(v2, v3, a);
  const u32 t3 = v3 >> a;
  u64 p = (u64)t0 * m;
  v0 = (u32)p;
  p = (u64)t1 * m + (p >> 32);
  v1 = (u32)p;
  p = (u64)t2 * m + (p >> 32);
  v2 = (u32)p;
  v3 = t3 * m + (u32)(p >> 32);
}

// ---------------------------------------------------------------------
// Generic L-limb values (wide range seeds, trajectory queries).
// ---------------------------------------------------------------------
template <int L>
struct Limbs {
  u32 w[L];
};

template <int L>
__device__ __forceinline__ bool limbs_lt(const Limbs<L>& a, const Limbs<L>& b) {
  bool lt = false, eq = true;
#pragma unroll
  for (int i = L - 1; i >= 0; i--) {
    lt = lt | (eq & (a.w[i] < b.w[i]));
    eq = eq & (a.w[i] == b.w[i]);
  }
  return lt;
}

// v <- (v >> a) * m, a <= 8, m = 3^a.  Returns false if the product left L limbs.
template <int L>
__device__ __forceinline__ bool odd_run_l(Limbs<L>& v, u32 a, u32 m) {
  u32 carry = 0;
#pragma unroll
  for (int i = 0; i < L; i++) {
    const u32 t = (i + 1 < L) ? __funnelshift_r(v.w[i], v.w[i + 1], a) : (v.w[i] >> a);
    const u64 p = (u64)t * m + carry;
    v.w[i] = (u32)p;
    carry = (u32)(p >> 32);
  }
  return carry == 0;
}

// m = v - 1 (v >= 1), exact with borrow.
template <int L>
__device__ __forceinline__ void dec_l(Limbs<L>& v) {
  u32 borrow = 1;
#pragma unroll
  for (int i = 0; i < L; i++) {
    const u32 x = v.w[i];
    v.w[i] = x - borrow;
    borrow = borrow & (x == 0);
  }
}
template <int L>
__device__ __forceinline__ void inc_l(Limbs<L>& v) {
  u32 carry = 1;
#pragma unroll
  for (int i = 0; i < L; i++) {
    const u32 x = v.w[i] + carry;
    carry = carry & (x == 0);
    v.w[i] = x;
  }
}
template <int L>
__device__ __forceinline__ void shr_l(Limbs<L>& v, u32 b) {  // b < 32
#pragma unroll
  for (int i = 0; i < L; i++)
    v.w[i] = (i + 1 < L) ? __funnelshift_r(v.w[i], v.w[i + 1], b) : (v.w[i] >> b);
}
template <int L>
__device__ __forceinline__ void shr_l_any(Limbs<L>& v, u32 s) {  // any s
  const u32 q = s >> 5, r = s & 31;
  Limbs<L> o;
#pragma unroll
  for (int i = 0; i < L; i++) {
    u32 lo = 0, hi = 0;
#pragma unroll
    for (int j = 0; j < L; j++) {
      if ((u32)j == i + q) lo = v.w[j];
      if ((u32)j == i + q + 1) hi = v.w[j];
    }
    o.w[i] = __funnelshift_r(lo, hi, r);
  }
  v = o;
}

// Number of significant bits of an L-limb value (0 for 0).
template <int L>
__device__ __forceinline__ u32 bitlen_l(const u32* w) {
  u32 bl = 0;
#pragma unroll
  for (int i = 0; i < L; i++)
    if (w[i]) bl = 32u * i + (32u - __clz(w[i]));
  return bl;
}

// ---------------------------------------------------------------------
// Monotone 64-bit key of an unsigned value: bits [63:54] = bit length,
// bits [53:0] = the top 54 bits (leading one included).  x < y implies
// key(x) <= key(y), and key(x) < key(y) implies x < y; decode() returns a
// value <= x.  Used as an atomicMax prefilter and as a threshold.
// ---------------------------------------------------------------------
template <int L>
__device__ __forceinline__ ull key_of(const u32* w) {
  u32 top = 0;
  int ti = -1;
#pragma unroll
  for (int i = 0; i < L; i++)
    if (w[i]) ti = i;
  if (ti < 0) return 0;
  u32 w2 = 0, w1 = 0, w0 = 0;
#pragma unroll
  for (int i = 0; i < L; i++) {
    if (i == ti) {
      w2 = w[i];
      w1 = (i > 0) ? w[i > 0 ? i - 1 : 0] : 0u;
      w0 = (i > 1) ? w[i > 1 ? i - 2 : 0] : 0u;
    }
  }
  top = __clz(w2);
  const ull bl = 32ull * ti + (32u - top);
  ull x = ((ull)w2 << 32) | w1;
  if (top) x = (x << top) | (w0 >> (32 - top));
  return (bl << 54) | (x >> 10);
}

// Lower-bound value of a key, as L limbs.
template <int L>
__device__ __forceinline__ void key_decode(ull key, u32* w) {
  const int bl = (int)(key >> 54);
  const ull m = key & ((1ull << 54) - 1);
  const int sh = bl - 54;  // value = m << sh (sh may be negative)
#pragma unroll
  for (int i = 0; i < L; i++) {
    const int d = 32 * i - sh;  // bit 32*i of the value is bit d of m
    u32 x;
    if (key == 0 || d >= 64 || d <= -32)
      x = 0;
    else if (d >= 0)
      x = (u32)(m >> d);
    else
      x = (u32)(m << (-d));
    w[i] = x;
  }
}

// ---------------------------------------------------------------------
// Record locks with a bounded spin: after LOCK_SPIN_LIMIT attempts the
// caller gives up and sets ERR_LOCK, so no kernel can wait forever.
// Callers serialise the lanes of a warp before taking a lock.
// ---------------------------------------------------------------------
__device__ __forceinline__ bool rec_lock(ReqRec* r) {
  for (u32 i = 0; i < LOCK_SPIN_LIMIT; i++) {
    if (atomicCAS(&r->lock, 0u, 1u) == 0u) {
      __threadfence();
      return true;
    }
    __nanosleep(64);
  }
  atomicOr(&r->errors, ERR_LOCK);
  return false;
}
__device__ __forceinline__ void rec_unlock(ReqRec* r) {
  __threadfence();
  atomicExch(&r->lock, 0u);
}

__device__ __forceinline__ bool seed_lt4(const u32* a, const volatile u32* b) {
  bool lt = false, eq = true;
#pragma unroll
  for (int i = 3; i >= 0; i--) {
    const u32 bi = b[i];
    lt = lt | (eq & (a[i] < bi));
    eq = eq & (a[i] == bi);
  }
  return lt;
}

// Offer (st, seed) as the maximum stopping time; ties go to the smaller seed.
static __device__ __noinline__ void rec_offer_st(ReqRec* r, ull st, const u32* seed) {
  const ull old = atomicMax(&r->st_key, st);
  if (old > st) return;
  if (!rec_lock(r)) return;
  volatile ReqRec* vr = r;
  const bool better = !(vr->valid & 1u) || st > vr->st || (st == vr->st && seed_lt4(seed, vr->st_seed));
  if (better) {
    vr->st = st;
#pragma unroll
    for (int i = 0; i < 4; i++) vr->st_seed[i] = seed[i];
    vr->valid = vr->valid | 1u;
  }
  rec_unlock(r);
}

// Offer (E, seed) as the maximum excursion (E has L <= 8 limbs).
template <int L>
static __device__ __noinline__ void rec_offer_e(ReqRec* r, const u32* E, const u32* seed) {
  const ull key = key_of<L>(E);
  const ull old = atomicMax(&r->e_key, key);
  if (old > key) return;
  if (!rec_lock(r)) return;
  volatile ReqRec* vr = r;
  bool lt = false, eq = true;  // E vs stored
#pragma unroll
  for (int i = 7; i >= 0; i--) {
    const u32 a = (i < L) ? E[i < L ? i : 0] : 0u;
    const u32 b = vr->E[i];
    lt = lt | (eq & (a < b));
    eq = eq & (a == b);
  }
  const bool better = !(vr->valid & 2u) || (!lt && !eq) || (eq && seed_lt4(seed, vr->E_seed));
  if (better) {
#pragma unroll
    for (int i = 0; i < 8; i++) vr->E[i] = (i < L) ? E[i < L ? i : 0] : 0u;
#pragma unroll
    for (int i = 0; i < 4; i++) vr->E_seed[i] = seed[i];
    vr->valid = vr->valid | 2u;
  }
  rec_unlock(r);
}

}  // namespace cz
