// noalloc.cu -- collatz_verify_pairs_noalloc: one batch of Step-1 pairs
// without allocating any memory.
//
// Some callers cannot allocate device memory when they verify a batch: a
// host application that hands this library device buffers out of its own
// memory pool and forbids other allocations, or a latency-bound loop in
// which cudaMalloc and cudaFree are not allowed because they can block and
// synchronize the whole device.  This entry point runs the same cases-mode
// kernel as collatz_verify_pairs, but the kernel's scratch (the result
// record, the pair counter and the overflow report) lives in a fixed
// file-scope device array instead of memory the context allocates on
// demand.  The caller passes the pairs already in device memory and gets
// the result back in host memory.
//
// Limits and rules:
//  * the scratch array is NOALLOC_SCRATCH_BYTES (64 KiB) on every GPU that
//    loads the library, held until the process exits;
//  * at most NOALLOC_OVERFLOW_MAX (4064) overflow seeds are reported per
//    call; a larger overflow_cap is rejected with COLLATZ_E_LIMIT;
//  * every call shares the array: the call clears it first, and calls that
//    overlap on the GPU (several host threads or streams at once) race;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress); make that first call before any stream capture.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "runtime.h"

namespace cz {

constexpr size_t NOALLOC_SCRATCH_BYTES = 64 * 1024;
constexpr size_t NOALLOC_REC_OFF = 0;       // ReqRec (136 bytes)
constexpr size_t NOALLOC_COUNTER_OFF = 256; // pair counter (u32)
constexpr size_t NOALLOC_OVCOUNT_OFF = 264; // overflow count (u64)
constexpr size_t NOALLOC_OVERFLOW_OFF = 512;
constexpr uint32_t NOALLOC_OVERFLOW_MAX = (uint32_t)((NOALLOC_SCRATCH_BYTES - NOALLOC_OVERFLOW_OFF) / 16);
static_assert(NOALLOC_OVERFLOW_MAX == 4064, "documented limit");
static_assert(sizeof(ReqRec) <= NOALLOC_COUNTER_OFF, "scratch layout");

// The scratch.  In host code this name is only a host-side stand-in for the
// device array; kernels get its device address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch per device, looked up once per device
// with that device current.
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[256];

static cudaError_t noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= 256) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_addr[device]);
  return cudaSuccess;
}

}  // namespace cz

using namespace cz;

#define NA_CK(c, expr)                                               \
  do {                                                               \
    cudaError_t e_ = (expr);                                         \
    if (e_ != cudaSuccess) return cz::set_cuda_error((c), e_, #expr); \
  } while (0)

extern "C" int collatz_verify_pairs_noalloc(collatz_ctx* c, uint32_t bigindex, const uint32_t* d_pairs,
                                            uint32_t npairs, collatz_case_result* out) {
  if (!c || !out || (npairs && !d_pairs)) return COLLATZ_E_ARG;
  if (c->ct.tpo + bigindex >= POW3_COUNT) return COLLATZ_E_ARG;
  if (out->overflow_cap > NOALLOC_OVERFLOW_MAX || (out->overflow_cap && !out->overflow_seeds)) {
    c->err = "collatz_verify_pairs_noalloc: overflow_cap " + std::to_string(out->overflow_cap) +
             " exceeds the allocation-free maximum of " + std::to_string(NOALLOC_OVERFLOW_MAX) + " seeds";
    return COLLATZ_E_LIMIT;
  }
  std::lock_guard<std::recursive_mutex> g(c->mu);
  uint32_t* ovbuf = out->overflow_seeds;
  const uint64_t ovcap = out->overflow_cap;
  std::memset(out, 0, sizeof *out);
  out->overflow_seeds = ovbuf;
  out->overflow_cap = ovcap;
  NA_CK(c, cudaSetDevice(c->device));
  unsigned char* base = nullptr;
  NA_CK(c, noalloc_scratch(c->device, &base));
  ReqRec* d_rec = reinterpret_cast<ReqRec*>(base + NOALLOC_REC_OFF);
  unsigned long long* d_ovcount = reinterpret_cast<unsigned long long*>(base + NOALLOC_OVCOUNT_OFF);
  // the previous call's contents stay in the array: clear the record and the counters
  NA_CK(c, cudaMemsetAsync(base, 0, NOALLOC_OVERFLOW_OFF, c->stream));
  if (npairs) {
    CasesArgs a;
    a.pairs = d_pairs;
    a.npairs = npairs;
    a.bigindex = (int)bigindex;
    a.bv = c->ct.bv;
    a.mod9 = c->ct.mod9;
    a.magic = c->ct.magic;
    a.pow3 = c->ct.pow3;
    a.mbi = c->ct.mbi;
    a.tpo = c->ct.tpo;
    a.pair_counter = reinterpret_cast<uint32_t*>(base + NOALLOC_COUNTER_OFF);
    a.rec = d_rec;
    a.overflow = reinterpret_cast<uint32_t*>(base + NOALLOC_OVERFLOW_OFF);
    a.overflow_cap = NOALLOC_OVERFLOW_MAX;
    a.overflow_count = d_ovcount;
    a.iter_cap = c->iter_cap;
    a.multi = 0;
    int bps = 0;
    if (cases_occupancy(c->cases_variant, &bps) != cudaSuccess || bps <= 0) bps = 1;
    NA_CK(c, cudaEventRecord(c->ev[0], c->stream));
    NA_CK(c, launch_cases(a, c->cases_variant, (uint32_t)(bps * c->sm_count), c->stream));
    NA_CK(c, cudaEventRecord(c->ev[1], c->stream));
  }
  ReqRec r;
  unsigned long long nov = 0;
  NA_CK(c, cudaMemcpyAsync(&r, d_rec, sizeof r, cudaMemcpyDeviceToHost, c->stream));
  NA_CK(c, cudaMemcpyAsync(&nov, d_ovcount, sizeof nov, cudaMemcpyDeviceToHost, c->stream));
  NA_CK(c, cudaStreamSynchronize(c->stream));
  if (npairs) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    out->device_ms = ms;
    if (bigindex < 16) {
      out->pairs = npairs;
      out->launches = 1;
    } else {
      out->cpu_pairs = npairs;
    }
  }
  out->hash = r.hash;
  out->seeds_checked = r.seeds;
  out->n_overflow = nov;
  out->errors = r.errors;
  if (r.valid & 2u) {
    std::memcpy(out->max_excursion, r.E, sizeof out->max_excursion);
    std::memcpy(out->max_excursion_seed, r.E_seed, sizeof out->max_excursion_seed);
  }
  if (r.valid & 1u) {
    out->max_stopping_time = r.st;
    std::memcpy(out->max_stopping_time_seed, r.st_seed, sizeof out->max_stopping_time_seed);
  }
  const uint64_t have = std::min<uint64_t>(std::min<uint64_t>(nov, NOALLOC_OVERFLOW_MAX), ovcap);
  if (have) {
    // copy straight into the caller's buffer, then sort in place (no allocation)
    NA_CK(c, cudaMemcpy(out->overflow_seeds, base + NOALLOC_OVERFLOW_OFF, 16 * have, cudaMemcpyDeviceToHost));
    struct Seed4 {
      uint32_t w[4];
    };
    Seed4* s = reinterpret_cast<Seed4*>(out->overflow_seeds);
    std::sort(s, s + have, [](const Seed4& x, const Seed4& y) {
      for (int i = 3; i >= 0; i--)
        if (x.w[i] != y.w[i]) return x.w[i] < y.w[i];
      return false;
    });
  }
  if (r.errors) {
    c->err = "device error bits 0x" + std::to_string(r.errors);
    return COLLATZ_E_DEVICE;
  }
  return COLLATZ_OK;
}
