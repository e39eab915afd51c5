// runtime.h -- host runtime shared by api.cu and server.cpp.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/collatz.h"
#include "kernels.h"
#include "rec.h"
#include "step1.h"
#include "tables.h"

namespace cz {

// Device buffer that only grows.
struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) n = bytes;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

// Pinned host buffer that only grows.
struct HostBuf {
  void* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMallocHost(&p, bytes);
    if (e == cudaSuccess) n = bytes;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

// Makes a device current for the lifetime of the object and then restores
// the device that was current for the calling thread, so that a library call
// does not change the caller's current device.
struct DeviceScope {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) err = cudaSetDevice(dev);
  }
  ~DeviceScope() {
    int now = -1;
    if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;
};

// "0x" followed by the value in upper-case hexadecimal.
inline std::string hex_u32(uint32_t x) {
  static const char* d = "0123456789ABCDEF";
  std::string s = "0x";
  bool lead = true;
  for (int i = 28; i >= 0; i -= 4) {
    const uint32_t n = (x >> i) & 15u;
    if (lead && n == 0 && i) continue;
    lead = false;
    s += d[n];
  }
  return s;
}

constexpr uint32_t WIDEN_CAP = 1u << 16;
constexpr uint32_t OVERFLOW_CAP = 1u << 16;
constexpr uint32_t CASE_BATCH = 1u << 20;  // pairs per device batch in run_case

struct RangeTables {
  RangeTable dev;
  std::vector<uint64_t> residues;  // host copy for k <= 28 (partial-block bounds)
};

}  // namespace cz

struct collatz_ctx {
  collatz_config cfg;
  int device = 0, sm_count = 0, sm_clock_khz = 0;
  cudaStream_t own_stream = nullptr, stream = nullptr, copy_stream = nullptr;
  cz::CaseTables ct;
  std::map<uint32_t, cz::RangeTables> rt;
  int cases_variant = 4, range_variant = 0;
  // 64-bit range kernel: its variant, and the limb-width cutoff -- launches whose seeds
  // all have at most range64_bits bits run it, the others run the four-limb kernel
  int range64_variant = 0;
  uint32_t range64_bits = 48;
  // resident blocks per SM of each range-kernel variant (0: not asked yet)
  int occ_range[8] = {}, occ_range64[8] = {};
  uint32_t iter_cap = 1u << 16;
  // scratch for the synchronous calls
  cz::DevBuf d_rec, d_counter, d_overflow, d_ovcount, d_pairs[2], d_segs, d_widen, d_widen2, d_wcount;
  cz::HostBuf h_rec, h_pairs;
  // one-shot range batches (collatz_verify_batch / collatz_verify_range)
  cz::DevBuf d_recs, d_rcursor, d_first;  // d_first: per request, its first segment (threshold scouts)
  cz::HostBuf h_segs, h_recs;
  std::vector<cz::RangeSeg> range_segs;
  cz::DevBuf t_seeds, t_st, t_exc, t_status, t_idx[2], t_cnt;
  // device Step 1: frontier (ping-pong), per-node leaf offsets and counts,
  // counters, pending-sibling stack
  cz::DevBuf s1_front[2], s1_off, s1_cnt, s1_scal, s1_stk_num, s1_stk_meta, s1_hist;
  cz::HostBuf h_s1;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  std::recursive_mutex mu;
  std::string err;
};

namespace cz {
int set_cuda_error(collatz_ctx* c, cudaError_t e, const char* where);

// Bit length of the largest seed of a range request (of its offset when it is empty).
inline uint32_t range_seed_bits(const collatz_range& r) {
  unsigned __int128 top = ((unsigned __int128)r.offset[1] << 64) | r.offset[0];
  if (r.size) top += r.size - 1;
  uint32_t b = 0;
  while (top) {
    top >>= 1;
    b++;
  }
  return b;
}
int get_range_tables(collatz_ctx* c, uint32_t k, RangeTables** out, bool negative = false);
// Launches the range kernel for a on stream s: the 64-bit kernel when every
// seed of the launch has at most c->range64_bits bits (positive variant),
// else the four-limb kernel; grid = resident blocks per SM x SMs.  stats:
// the diagnostics form of the chosen kernel.
cudaError_t range_kernel_launch(collatz_ctx* c, const RangeArgs& a, bool stats, cudaStream_t s);
int lower_range(collatz_ctx* c, const collatz_range& r, uint32_t req, const RangeTables& T,
                std::vector<RangeSeg>& segs, unsigned long long& items);
void rec_to_range_result(const ReqRec& r, collatz_range_result* out);
// Applies cached autotuner choices to a new context (tune.cu).
void tune_on_create(collatz_ctx* c);
}  // namespace cz
