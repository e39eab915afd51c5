/*
 * CPU stand-in for the handful of CUDA runtime names that
 * collatz_cudav7.cu uses, so that the reference program compiles with g++
 * and runs sequentially on the host (oracle/build_ref.sh).
 *
 * TEST INFRASTRUCTURE ONLY: the binaries built with it live in
 * oracle/_ref/ and serve as the checker that pins the oracle.
 *
 * Sequential emulation is exact for compute_kernel: its only warp
 * intrinsic, __any_sync (cu:296, 335), guards a per-thread branch, and the
 * per-thread hashes are combined with XOR (cu:407-409).
 */
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#define __global__
#define __constant__
#define __device__
#define __host__

struct shim_dim3 {
  unsigned x, y, z;
};
static thread_local shim_dim3 threadIdx, blockIdx, blockDim;

typedef int cudaError_t;
enum { cudaSuccess = 0 };
enum { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };
enum { cudaDeviceScheduleBlockingSync = 4 };

static inline int cudaSetDeviceFlags(unsigned) { return 0; }
template <class T>
static inline int cudaMalloc(T **p, size_t n) {
  *p = (T *)std::malloc(n ? n : 1);
  return 0;
}
static inline int cudaMemcpy(void *d, const void *s, size_t n, int) {
  std::memcpy(d, s, n);
  return 0;
}
static inline int cudaFree(void *p) {
  std::free(p);
  return 0;
}
static inline int cudaGetLastError() { return 0; }
static inline int cudaDeviceSynchronize() { return 0; }
static inline const char *cudaGetErrorString(int) { return "no error"; }

static inline uint32_t __brev(uint32_t x) {
  uint32_t r = 0;
  for (int i = 0; i < 32; i++) r |= ((x >> i) & 1u) << (31 - i);
  return r;
}
static inline int __clz(uint32_t x) { return x ? __builtin_clz(x) : 32; }
static inline int __ffs(uint32_t x) { return __builtin_ffs((int)x); }
static inline uint32_t __funnelshift_r(uint32_t lo, uint32_t hi, uint32_t sh) {
  return (uint32_t)(((((uint64_t)hi) << 32) | lo) >> (sh & 31));
}
static inline bool __any_sync(unsigned, bool p) { return p; }
static inline uint32_t atomicXor(uint32_t *a, uint32_t v) {
  uint32_t o = *a;
  *a ^= v;
  return o;
}

/* seeds-checked counter: build_ref.sh inserts shim_count_seeds(alength)
 * right after Step 2 of compute_kernel; printed to stderr at exit. */
static unsigned long long shim_seed_count;
static inline void shim_count_seeds(unsigned n) { shim_seed_count += n; }
struct shim_report_t {
  ~shim_report_t() {
    if (!std::getenv("SHIM_QUIET")) std::fprintf(stderr, "shim seeds = %llu\n", shim_seed_count);
  }
};
static shim_report_t shim_report_instance;

/* kernel launch <<<grid, block>>> replaced by a sequential loop */
#define SHIM_LAUNCH(grid, block, fn, ...)                                  \
  do {                                                                     \
    blockDim.x = (block);                                                  \
    for (unsigned b_ = 0; b_ < (unsigned)(grid); b_++)                     \
      for (unsigned t_ = 0; t_ < (unsigned)(block); t_++) {                \
        blockIdx.x = b_;                                                   \
        threadIdx.x = t_;                                                  \
        fn(__VA_ARGS__);                                                   \
      }                                                                    \
  } while (0)
