// step1_dev.cu -- Step 1 of the reference's Algorithm 1 (search1,
// collatz_cudav7.cu:497-563) on the device: the bit-by-bit tree over the
// low N-A bits of n, pruned by the induction sieve (cu:507) and the mod-3
// path-merging sieve (cu:509-511), whose leaves (sigfig == N-A) are the
// (base, number) pairs that the cases kernel verifies.
//
// The host cuts the case's tree into a few thousand subtree roots.  Then:
//   k_step1_expand  one tree level per launch, breadth first: each node
//                   writes its surviving children (warp-aggregated append).
//                   The host picks the number of levels so that the output
//                   never exceeds the frontier buffer (each level at most
//                   doubles), so no level needs a host round trip.
//   k_step1_walk    depth first below the frontier, one subtree per lane
//                   (a warp takes 32 consecutive frontier nodes at a time).
//                   The count pass gives each frontier node its leaf count
//                   and a first leaf index (one atomic per warp) and counts
//                   the leaves per bigindex; the emit pass writes the pairs
//                   whose leaf index lies in a window [w_lo, w_hi), so the
//                   pairs of any tree go to the device in bounded chunks.
// Each lane keeps at most one pending sibling per tree level (the right
// child, base | 1 << sigfig): its state lives in a global stack laid out
// [level][thread], and its base is rebuilt from the current path on pop.
//
// Line batches: the roots may be many cases_* lines at different sigfigs.
// A node's sigfig word is sigfig | line << 8; a leaf reached before the last
// breadth-first level passes through the later levels unchanged; the count
// pass counts leaves per (line, bigindex), one line per block in shared
// memory and the others with global atomics; a pair carries
// bigindex | line << 8 in base limb 3.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace cz {

typedef unsigned __int128 u128d;

namespace {

constexpr uint32_t NUMER = 306, DENOM = 485;  // cu:49-50

__device__ __forceinline__ u128d mk(unsigned long long lo, unsigned long long hi) {
  return ((u128d)hi << 64) | lo;
}

// Entry tests of search1 (cu:507-511), in 32-bit unsigned arithmetic like the
// reference (sigfig - 1 and threepower - 1 wrap at 0).
__device__ __forceinline__ bool s1_pass(uint32_t sig, uint32_t tp, uint32_t ne) {
  if (DENOM * tp <= NUMER * sig) return false;
  if (ne >= 2u && (ne & 1u) == 0u && NUMER * (sig - 1u) >= DENOM * (tp - 1u)) return false;
  return true;
}

struct Kid {
  u128d num;
  uint32_t tp, de, ne;
  bool ok;
};

// The two children of an inner node in the reference's visiting order
// (cu:543-561).  The second child is always the one with bit sigfig set.
__device__ __forceinline__ void s1_children(u128d num, uint32_t sig, uint32_t tp, uint32_t de, uint32_t ne,
                                            const u128d* p3, Kid& a, Kid& b) {
  const uint32_t dip = (NUMER * (sig + 1u) >= DENOM * tp) ? 1u : 0u;
  const u128d B = num + p3[tp & 127u];
  if (((uint32_t)num & 1u) == 0u) {
    a.num = num + (num >> 1);
    a.tp = tp + 1u;
    a.de = (de | dip) & ~2u;
    a.ne = 0u;
    a.ok = true;
    b.num = (B >> 1) + 1u;
    b.tp = tp;
    b.de = de << 1;
    b.ne = ne + 1u;
    b.ok = de < 2u;
  } else {
    a.num = (num >> 1) + 1u;
    a.tp = tp;
    a.de = de << 1;
    a.ne = ne + 1u;
    a.ok = de < 2u;
    b.num = B + (B >> 1);
    b.tp = tp + 1u;
    b.de = (de | dip) & ~2u;
    b.ne = 0u;
    b.ok = true;
  }
  a.ok = a.ok && s1_pass(sig + 1u, a.tp, a.ne);
  b.ok = b.ok && s1_pass(sig + 1u, b.tp, b.ne);
}

// THREEPOWERS (cu:104-105): 3^i mod 2^128, i < 128.
__device__ __forceinline__ void init_pow3(u128d* p3) {
  for (uint32_t i = threadIdx.x; i < 128u; i += blockDim.x) {
    u128d r = 1, b = 3;
    for (uint32_t e = i; e; e >>= 1) {
      if (e & 1u) r *= b;
      b *= b;
    }
    p3[i] = r;
  }
}

// sig: sigfig (< 256); line: the node's line in a line batch (0 otherwise).
__device__ __forceinline__ void load_node(const S1Node* p, u128d& base, u128d& num, uint32_t& sig, uint32_t& tp,
                                          uint32_t& de, uint32_t& ne, uint32_t& line) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  const uint4 x = q[0], y = q[1], z = q[2];
  base = mk(((unsigned long long)x.y << 32) | x.x, ((unsigned long long)x.w << 32) | x.z);
  num = mk(((unsigned long long)y.y << 32) | y.x, ((unsigned long long)y.w << 32) | y.z);
  sig = z.x & 0xFFu;
  line = z.x >> 8;
  tp = z.y;
  de = z.z;
  ne = z.w;
}

__device__ __forceinline__ void store_node(S1Node* p, u128d base, u128d num, uint32_t sig, uint32_t tp, uint32_t de,
                                           uint32_t ne, uint32_t line) {
  uint4* q = reinterpret_cast<uint4*>(p);
  q[0] = make_uint4((uint32_t)base, (uint32_t)(base >> 32), (uint32_t)(base >> 64), (uint32_t)(base >> 96));
  q[1] = make_uint4((uint32_t)num, (uint32_t)(num >> 32), (uint32_t)(num >> 64), (uint32_t)(num >> 96));
  q[2] = make_uint4(sig | (line << 8), tp, de, ne);
}

}  // namespace

// One breadth-first level: frontier (in, *in_count) -> children (out,
// *out_count).  A leaf (sigfig == N-A) is copied through unchanged.
__global__ void __launch_bounds__(256) k_step1_expand(const Step1Args A) {
  __shared__ u128d p3[128];
  const uint32_t n = *A.in_count;
  if (blockIdx.x * blockDim.x >= n) return;  // whole block past the frontier
  init_pow3(p3);
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u;
  Kid a, b;
  a.ok = b.ok = false;
  u128d base = 0;
  uint32_t sig = 0, line = 0;
  bool leaf = false;
  if (i < n) {
    u128d num;
    uint32_t tp, de, ne;
    load_node(A.in + i, base, num, sig, tp, de, ne, line);
    if (sig == A.mbi) {  // pass the leaf through as the first "child"
      leaf = true;
      a.num = num;
      a.tp = tp;
      a.de = de;
      a.ne = ne;
      a.ok = true;
    } else {
      s1_children(num, sig, tp, de, ne, p3, a, b);
    }
  }
  const uint32_t k = (uint32_t)a.ok + (uint32_t)b.ok;
  uint32_t incl = k;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(FULL, incl, d);
    if (lane >= (uint32_t)d) incl += t;
  }
  uint32_t wbase = 0;
  if (lane == 31u && incl) wbase = atomicAdd(A.out_count, incl);
  wbase = __shfl_sync(FULL, wbase, 31);
  uint32_t o = wbase + incl - k;
  if (a.ok) store_node(A.out + o++, base, a.num, leaf ? sig : sig + 1u, a.tp, a.de, a.ne, line);
  if (b.ok) store_node(A.out + o, base | ((u128d)1 << sig), b.num, sig + 1u, b.tp, b.de, b.ne, line);
}

// Depth-first walk below the frontier; see the file comment.
template <bool EMIT>
__global__ void __launch_bounds__(128) k_step1_walk(const Step1Args A) {
  __shared__ u128d p3[128];
  __shared__ unsigned long long hist[17];
  __shared__ uint32_t s_line;  // line batches: the line whose leaves this block counts in `hist`
  init_pow3(p3);
  if (threadIdx.x < 17u) hist[threadIdx.x] = 0ull;
  const uint32_t n = *A.in_count;
  if (threadIdx.x == 0)  // a frontier node's line (one line per block is counted in shared memory)
    s_line = (!EMIT && A.hist_lines && n) ? (A.in[min(blockIdx.x * 32u, n - 1u)].sig >> 8) : 0u;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t T = A.nthreads;
  for (;;) {
    uint32_t wb = 0;
    if (lane == 0u) wb = atomicAdd(A.cursor, 32u);
    wb = __shfl_sync(FULL, wb, 0);
    if (wb >= n) break;
    const uint32_t i = wb + lane;
    unsigned long long cnt = 0, off = 0;
    bool go = i < n;
    if (EMIT && go) {
      off = A.off[i];
      go = off < A.w_hi && off + A.cnt[i] > A.w_lo;
    }
    if (go) {
      u128d base, num;
      uint32_t sig, tp, de, ne, line;
      load_node(A.in + i, base, num, sig, tp, de, ne, line);
      const uint32_t s0 = sig;
      unsigned long long pend_lo = 0, pend_hi = 0;  // bit l: a pending node at sigfig s0 + 1 + l
      for (;;) {
        bool pop = false;
        if (sig == A.mbi) {
          const uint32_t bi = tp - A.tpo;
          if (EMIT) {
            const unsigned long long idx = off + cnt;
            if (idx >= A.w_lo) {
              uint4* q = reinterpret_cast<uint4*>(A.pairs + 8ull * (idx - A.w_lo));
              q[0] = make_uint4((uint32_t)base, (uint32_t)(base >> 32), (uint32_t)(base >> 64), bi | (line << 8));
              q[1] = make_uint4((uint32_t)num, (uint32_t)(num >> 32), (uint32_t)(num >> 64),
                                (uint32_t)(num >> 96));
            }
          } else if (A.hist_lines && line != s_line) {
            atomicAdd(&A.hist_lines[17ull * line + (bi < 16u ? bi : 16u)], 1ull);
          } else {
            atomicAdd(&hist[bi < 16u ? bi : 16u], 1ull);
          }
          cnt++;
          if (EMIT && off + cnt >= A.w_hi) break;  // the rest lies past the window
          pop = true;
        } else {
          Kid a, b;
          s1_children(num, sig, tp, de, ne, p3, a, b);
          if (a.ok) {
            if (b.ok) {
              const uint32_t l = sig - s0;
              const size_t at = (size_t)l * T + tid;
              A.stk_num[at] = make_ulonglong2((unsigned long long)b.num, (unsigned long long)(b.num >> 64));
              A.stk_meta[at] = make_uint4(b.tp, b.de, b.ne, 0u);
              if (l < 64u) pend_lo |= 1ull << l;
              else pend_hi |= 1ull << (l - 64u);
            }
            num = a.num;
            tp = a.tp;
            de = a.de;
            ne = a.ne;
            sig++;
          } else if (b.ok) {
            base |= (u128d)1 << sig;
            num = b.num;
            tp = b.tp;
            de = b.de;
            ne = b.ne;
            sig++;
          } else {
            pop = true;
          }
        }
        if (pop) {
          if (!(pend_lo | pend_hi)) break;
          uint32_t l;
          if (pend_hi) {
            l = 127u - (uint32_t)__clzll((long long)pend_hi);
            pend_hi &= ~(1ull << (l - 64u));
          } else {
            l = 63u - (uint32_t)__clzll((long long)pend_lo);
            pend_lo &= ~(1ull << l);
          }
          const size_t at = (size_t)l * T + tid;
          const ulonglong2 v = A.stk_num[at];
          const uint4 m = A.stk_meta[at];
          const uint32_t pb = s0 + l;  // parent's sigfig: the bit the pending child sets
          base = (base & (((u128d)1 << pb) - 1u)) | ((u128d)1 << pb);
          num = mk(v.x, v.y);
          tp = m.x;
          de = m.y;
          ne = m.z;
          sig = pb + 1u;
        }
      }
    }
    if (!EMIT) {
      unsigned long long incl = cnt;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long t = __shfl_up_sync(FULL, incl, d);
        if (lane >= (uint32_t)d) incl += t;
      }
      unsigned long long base0 = 0;
      if (lane == 31u && incl) base0 = atomicAdd(A.total, incl);
      base0 = __shfl_sync(FULL, base0, 31);
      if (i < n) {
        A.off[i] = base0 + incl - cnt;
        A.cnt[i] = cnt;
      }
    }
  }
  if (!EMIT) {
    __syncthreads();
    if (threadIdx.x < 17u && hist[threadIdx.x])
      atomicAdd((A.hist_lines ? A.hist_lines + 17ull * s_line : A.hist) + threadIdx.x, hist[threadIdx.x]);
  }
}

cudaError_t launch_step1_expand(const Step1Args& a, uint32_t bound, cudaStream_t st) {
  if (bound == 0) return cudaSuccess;
  k_step1_expand<<<(bound + 255u) / 256u, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_step1_walk(const Step1Args& a, bool emit, cudaStream_t st) {
  const uint32_t grid = a.nthreads / 128u;
  if (emit) k_step1_walk<true><<<grid, 128, 0, st>>>(a);
  else k_step1_walk<false><<<grid, 128, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace cz
