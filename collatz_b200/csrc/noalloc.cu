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
//  * every call looks up the array's device address (cudaGetSymbolAddress)
//    with the context's device current, so the address stays right after the
//    host application resets or recreates the primary context; the first call
//    on a device also loads the module, so make it before any stream capture;
//  * when the caller's overflow_cap is smaller than the number of overflow
//    seeds, the smallest overflow_cap seeds are returned, as by
//    collatz_verify_pairs (the device list is read in fixed-size pieces
//    through a stack buffer and kept in a bounded heap in the caller's
//    buffer, so no host memory is allocated either).
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

// Device address of g_noalloc_scratch on the current device.
static cudaError_t noalloc_scratch(unsigned char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<unsigned char*>(p);
  return cudaSuccess;
}

// An overflow seed as the kernel reports it: limbs 0..2 of a 96-bit value
// (limb 3 unused), ordered by value.
struct Seed4 {
  uint32_t w[4];
};
static bool seed_less(const Seed4& x, const Seed4& y) {
  for (int i = 2; i >= 0; i--)
    if (x.w[i] != y.w[i]) return x.w[i] < y.w[i];
  return false;
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
  if (bigindex >= POW3_COUNT || (uint64_t)c->ct.tpo + bigindex >= POW3_COUNT) return COLLATZ_E_ARG;
  if (out->overflow_cap && !out->overflow_seeds) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  if (out->overflow_cap > NOALLOC_OVERFLOW_MAX) {
    c->err = "collatz_verify_pairs_noalloc: overflow_cap " + std::to_string(out->overflow_cap) +
             " exceeds the allocation-free maximum of " + std::to_string(NOALLOC_OVERFLOW_MAX) + " seeds";
    return COLLATZ_E_LIMIT;
  }
  uint32_t* ovbuf = out->overflow_seeds;
  const uint64_t ovcap = out->overflow_cap;
  std::memset(out, 0, sizeof *out);
  out->overflow_seeds = ovbuf;
  out->overflow_cap = ovcap;
  DeviceScope dev_scope(c->device);
  NA_CK(c, dev_scope.err);
  unsigned char* base = nullptr;
  NA_CK(c, noalloc_scratch(&base));
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
  const uint64_t have = std::min<uint64_t>(nov, NOALLOC_OVERFLOW_MAX);
  const uint64_t keep = std::min<uint64_t>(have, ovcap);
  if (keep) {
    // the smallest `keep` of the `have` device entries: read them in pieces through a
    // stack buffer into a max-heap of at most `keep` seeds held in the caller's buffer,
    // then sort the heap (no allocation)
    Seed4* heap = reinterpret_cast<Seed4*>(out->overflow_seeds);
    uint64_t n = 0;
    Seed4 piece[128];
    for (uint64_t i = 0; i < have; i += 128) {
      const uint64_t m = std::min<uint64_t>(128, have - i);
      NA_CK(c, cudaMemcpy(piece, base + NOALLOC_OVERFLOW_OFF + 16 * i, 16 * m, cudaMemcpyDeviceToHost));
      for (uint64_t j = 0; j < m; j++) {
        piece[j].w[3] = 0;
        if (n < keep) {
          heap[n++] = piece[j];
          std::push_heap(heap, heap + n, seed_less);
        } else if (seed_less(piece[j], heap[0])) {
          std::pop_heap(heap, heap + n, seed_less);
          heap[n - 1] = piece[j];
          std::push_heap(heap, heap + n, seed_less);
        }
      }
    }
    std::sort_heap(heap, heap + n, seed_less);
  }
  if (r.errors) {
    c->err = "device error bits " + hex_u32(r.errors);
    return COLLATZ_E_DEVICE;
  }
  return COLLATZ_OK;
}
