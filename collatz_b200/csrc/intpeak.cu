// intpeak.cu -- measured 32-bit integer peak of this device (collatz_int_peak).
//
// The hot kernels are integer-issue bound, and the device has no published
// integer throughput to divide by.  This loop measures one: every SM full of
// warps (8 blocks x 256 threads), each thread running 8 independent chains
// of dependent 32-bit operations, timed with CUDA events.  Two mixes:
//   mix 0 (ALU): funnel shift, 3-input add, 3-input logic op per link;
//   mix 1 (kernel mix): funnel shift, 3-input add, multiply-add per link --
//     two ALU-pipe operations to one FMA-pipe multiply-add, the proportion
//     the run arithmetic of the range and cases kernels has.
// One operation per link step is one instruction (the instruction count is
// checked with ncu's sm__inst_executed).  Block 0 also reads the SM clock
// and the global timer at both ends, so the result carries the clock the
// loop actually ran at and a per-clock rate that scales to other clocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "runtime.h"

using namespace cz;

namespace {

constexpr uint32_t PEAK_BLOCK = 256, PEAK_BLOCKS_PER_SM = 8, PEAK_CHAINS = 8, PEAK_OPS_PER_LINK = 3;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <int MIX>
__global__ void __launch_bounds__(PEAK_BLOCK, PEAK_BLOCKS_PER_SM)
    k_int_peak(uint32_t iters, uint32_t m, uint32_t c, uint32_t* out, unsigned long long* clk) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t x[PEAK_CHAINS], y[PEAK_CHAINS];
#pragma unroll
  for (uint32_t j = 0; j < PEAK_CHAINS; j++) {
    x[j] = tid * (2u * j + 1u) + c;
    y[j] = x[j] ^ (0x9E3779B9u * (j + 1u));
  }
  const bool timer = (tid == 0);
  unsigned long long c0 = 0, t0 = 0;
  if (timer) {
    t0 = global_ns();
    c0 = clock64();
  }
#pragma unroll 4
  for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
    for (uint32_t j = 0; j < PEAK_CHAINS; j++) {
      x[j] = __funnelshift_r(x[j], y[j], 7);  // shift (ALU)
      y[j] = y[j] + x[j] + c;                 // 3-input add (ALU)
      if (MIX == 0)
        x[j] = x[j] ^ (y[j] & m);             // 3-input logic (ALU)
      else
        x[j] = x[j] * m + y[j];               // multiply-add (FMA pipe)
    }
  }
  if (timer) {
    clk[0] = clock64() - c0;
    clk[1] = global_ns() - t0;
  }
  uint32_t h = 0;
#pragma unroll
  for (uint32_t j = 0; j < PEAK_CHAINS; j++) h ^= x[j] + y[j];
  out[tid] = h;
}

}  // namespace

extern "C" int collatz_int_peak(collatz_ctx* ctx, int mix, collatz_int_peak_t* out) {
  if (!ctx || !out || (mix != 0 && mix != 1)) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(ctx->mu);
  std::memset(out, 0, sizeof *out);
  DeviceScope dev_scope(ctx->device);
  cudaError_t e = dev_scope.err;
  const uint32_t grid = (uint32_t)ctx->sm_count * PEAK_BLOCKS_PER_SM;
  const uint32_t threads = grid * PEAK_BLOCK;
  // 2^17 iterations: 24 operations per iteration and thread, about 30 ms per launch
  const uint32_t iters = 1u << 17;
  uint32_t* d_out = nullptr;
  unsigned long long* d_clk = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (!e) e = cudaMalloc(&d_out, (size_t)threads * sizeof(uint32_t));
  if (!e) e = cudaMalloc(&d_clk, 2 * sizeof(unsigned long long));
  if (!e) e = cudaEventCreate(&ev[0]);
  if (!e) e = cudaEventCreate(&ev[1]);
  float best = 0.0f;
  unsigned long long best_clk[2] = {0, 0};
  // one warm-up launch, then the fastest of 3 timed launches
  for (int rep = 0; rep < 4 && !e; rep++) {
    e = cudaEventRecord(ev[0], ctx->stream);
    if (!e) {
      if (mix == 0)
        k_int_peak<0><<<grid, PEAK_BLOCK, 0, ctx->stream>>>(iters, 0x5bd1e995u, 0x1234567u, d_out, d_clk);
      else
        k_int_peak<1><<<grid, PEAK_BLOCK, 0, ctx->stream>>>(iters, 0x5bd1e995u, 0x1234567u, d_out, d_clk);
      e = cudaGetLastError();
    }
    if (!e) e = cudaEventRecord(ev[1], ctx->stream);
    if (!e) e = cudaEventSynchronize(ev[1]);
    float ms = 0.0f;
    if (!e) e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
    unsigned long long h_clk[2] = {0, 0};
    if (!e) e = cudaMemcpy(h_clk, d_clk, sizeof h_clk, cudaMemcpyDeviceToHost);
    if (!e && rep > 0 && (best == 0.0f || ms < best)) {
      best = ms;
      best_clk[0] = h_clk[0];
      best_clk[1] = h_clk[1];
    }
  }
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  if (d_out) cudaFree(d_out);
  if (d_clk) cudaFree(d_clk);
  if (e) return set_cuda_error(ctx, e, "collatz_int_peak");
  out->ops = (uint64_t)threads * iters * PEAK_CHAINS * PEAK_OPS_PER_LINK;
  out->ms = best;
  out->ops_per_s = (double)out->ops / (best * 1e-3);
  out->sm_mhz = best_clk[1] ? (double)best_clk[0] * 1e3 / (double)best_clk[1] : 0.0;
  out->ops_per_clk_sm = out->sm_mhz > 0.0 ? out->ops_per_s / (out->sm_mhz * 1e6 * ctx->sm_count) : 0.0;
  out->sm_count = (uint32_t)ctx->sm_count;
  out->mix = (uint32_t)mix;
  return COLLATZ_OK;
}
