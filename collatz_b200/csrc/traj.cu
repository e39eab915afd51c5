// traj.cu -- per-seed trajectory queries: for arbitrary seeds up to 256
// bits, the exact stopping time sigma(n) (least k >= 1 with T^k(n) < n) and
// the maximum excursion E(n) = max_{k <= sigma} T^k(n).
//
// One seed per lane with per-lane dynamic fetch, so the warp stays busy
// while seeds of very different lengths finish.  The host sorts seeds by
// bit length into limb classes (L = 4, 6, 8, 12, 16) and one launch serves
// every class; a seed whose value could leave L limbs is run again by its
// thread with the next width.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace cz {

template <int L>
__device__ __forceinline__ void load_seed(const u32* __restrict__ s, Limbs<L>& n) {
#pragma unroll
  for (int j = 0; j < L; j++) n.w[j] = (j < 8) ? s[j < 8 ? j : 0] : 0u;
}

// ------------------------------------------------------------------
// All limb classes in one launch.  index holds the seed ids sorted by class
// (class j at [cstart[j], cstart[j + 1]); classes of 4, 6, 8, 12, 16 limbs);
// every lane takes the next slot from one cursor and runs that seed with its
// class's width.  A seed whose value could leave L limbs is run again from
// the start with the next width, by the same thread; past 16 limbs its status
// is 2.
// ------------------------------------------------------------------
template <int L>
struct WiderLimbs {
  static constexpr int value = L == 4 ? 6 : L == 6 ? 8 : L == 8 ? 12 : L == 12 ? 16 : 0;
};

template <int L>
__device__ __noinline__ void traj_seed(const TrajAllArgs& A, u32 sid, const u32* s_pow3) {
  Limbs<L> N, v, E;
  load_seed<L>(A.seeds + 8ull * sid, N);
  bool small = N.w[0] < 2u;
#pragma unroll
  for (int j = 1; j < L; j++) small = small & (N.w[j] == 0u);
  if (small) {  // n = 0, 1: no stopping time
    A.st[sid] = 0;
#pragma unroll
    for (int j = 0; j < 16; j++) A.exc[16ull * sid + j] = (j < L) ? N.w[j < L ? j : 0] : 0u;
    A.status[sid] = 1;
    return;
  }
  v = N;
  inc_l<L>(v);
  E = N;
  unsigned long long st = 0;
  for (u32 it = 0;; it++) {
    if (v.w[L - 1] >= (1u << 19)) {  // the next odd run could leave L limbs
      if constexpr (WiderLimbs<L>::value != 0) {
        traj_seed<WiderLimbs<L>::value>(A, sid, s_pow3);
      } else {
        A.st[sid] = 0;
#pragma unroll
        for (int j = 0; j < 16; j++) A.exc[16ull * sid + j] = 0u;
        A.status[sid] = 2;
      }
      return;
    }
    if (it >= A.iter_cap) {
      A.st[sid] = 0;
#pragma unroll
      for (int j = 0; j < 16; j++) A.exc[16ull * sid + j] = 0u;
      A.status[sid] = 3;
      return;
    }
    const u32 a = ctz32(v.w[0] | (1u << 8));
    odd_run_l<L>(v, a, s_pow3[a]);
    st += a;
    Limbs<L> x = v;
    dec_l<L>(x);
    if (limbs_lt<L>(E, x)) E = x;
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
      A.st[sid] = st + s;
#pragma unroll
      for (int j = 0; j < 16; j++) A.exc[16ull * sid + j] = (j < L) ? E.w[j < L ? j : 0] : 0u;
      A.status[sid] = 0;
      return;
    }
    st += b;
    v = w;
    inc_l<L>(v);
  }
}

__global__ void __launch_bounds__(128) k_traj_all(const TrajAllArgs A) {
  __shared__ u32 s_pow3[9];
  if (threadIdx.x < 9) {
    u32 p = 1;
    for (u32 i = 0; i < threadIdx.x; i++) p *= 3;
    s_pow3[threadIdx.x] = p;
  }
  __syncthreads();
  for (;;) {
    const u32 slot = atomicAdd(A.cursor, 1u);
    if (slot >= A.cstart[5]) break;
    const u32 sid = A.index[slot];
    if (slot < A.cstart[1])
      traj_seed<4>(A, sid, s_pow3);
    else if (slot < A.cstart[2])
      traj_seed<6>(A, sid, s_pow3);
    else if (slot < A.cstart[3])
      traj_seed<8>(A, sid, s_pow3);
    else if (slot < A.cstart[4])
      traj_seed<12>(A, sid, s_pow3);
    else
      traj_seed<16>(A, sid, s_pow3);
  }
}

cudaError_t launch_traj_all(const TrajAllArgs& a, u32 grid, cudaStream_t st) {
  k_traj_all<<<grid, 128, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace cz
