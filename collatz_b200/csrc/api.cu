// api.cu -- the C ABI of include/collatz.h: context, cases mode (host
// Step 1 feeding the GPU), range plans (lowered work lists + captured CUDA
// graphs), trajectory queries.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>
#include <cstdio>
#include <cstdlib>

#include "runtime.h"

using namespace cz;

static const size_t BV_WORDS_HOST = (1u << 19) + 32u;

#define CK(c, expr)                                                  \
  do {                                                               \
    cudaError_t e_ = (expr);                                         \
    if (e_ != cudaSuccess) return cz::set_cuda_error((c), e_, #expr); \
  } while (0)

namespace cz {

int set_cuda_error(collatz_ctx* c, cudaError_t e, const char* where) {
  if (c) c->err = std::string(where) + ": " + cudaGetErrorString(e);
  cudaGetLastError();
  return COLLATZ_E_CUDA;
}

static u128 u128_of(const uint64_t* x) { return ((u128)x[1] << 64) | x[0]; }

static void limbs4(u128 x, uint32_t* w) {
  for (int i = 0; i < 4; i++) w[i] = (uint32_t)(x >> (32 * i));
}

static int grid_for(collatz_ctx* c, int mode, int variant) {
  int bps = 0;
  cudaError_t e = mode == 0 ? cases_occupancy(variant, &bps) : range_occupancy(variant, &bps);
  if (e != cudaSuccess || bps <= 0) bps = 1;
  return bps * c->sm_count;
}

void rec_to_range_result(const ReqRec& r, collatz_range_result* out) {
  std::memset(out, 0, sizeof *out);
  out->seeds_checked = r.seeds;
  out->failures = r.failures;
  out->widened = r.widened;
  if (r.valid & 2u) {
    std::memcpy(out->max_excursion, r.E, sizeof r.E);
    std::memcpy(out->max_excursion_seed, r.E_seed, sizeof r.E_seed);
  }
  if (r.valid & 1u) {
    out->max_stopping_time = r.st;
    std::memcpy(out->max_stopping_time_seed, r.st_seed, sizeof r.st_seed);
  }
  out->errors = r.errors;
  out->status = r.errors ? COLLATZ_E_DEVICE : COLLATZ_OK;
}

// ---------------------------------------------------------------------
// Range tables and lowering of requests into work segments.
// ---------------------------------------------------------------------

int get_range_tables(collatz_ctx* c, uint32_t k, RangeTables** out, bool negative) {
  const uint32_t key = k | (negative ? 0x100u : 0u);
  auto it = c->rt.find(key);
  if (it != c->rt.end()) {
    *out = &it->second;
    return COLLATZ_OK;
  }
  RangeTables T;
  cudaError_t e = build_range_table(&T.dev, k, true, c->own_stream, negative);
  if (e != cudaSuccess) {
    free_range_table(&T.dev);
    return set_cuda_error(c, e, "build_range_table");
  }
  if (T.dev.violations) {
    c->err = "range sieve validation failed for k=" + std::to_string(k);
    free_range_table(&T.dev);
    return COLLATZ_E_DEVICE;
  }
  if (k <= 28 && T.dev.count) {
    std::vector<RangeEntry> h(T.dev.count);
    e = cudaMemcpy(h.data(), T.dev.table, sizeof(RangeEntry) * T.dev.count, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_cuda_error(c, e, "range table copy");
    T.residues.resize(T.dev.count);
    for (size_t i = 0; i < h.size(); i++) T.residues[i] = (uint64_t)h[i].r_lo | ((uint64_t)(h[i].meta & 0xFF) << 32);
  }
  auto ins = c->rt.emplace(key, std::move(T));
  *out = &ins.first->second;
  return COLLATZ_OK;
}

// index of the first survivor >= r within mod-9 class cl of the class-major table
static int lower_bound_res(collatz_ctx* c, const RangeTables& T, uint32_t cl, uint64_t r, uint32_t* out) {
  const uint64_t b = T.dev.cls[cl], e = T.dev.cls[cl + 1];
  if (r == 0 || b == e) {
    *out = (uint32_t)b;
    return COLLATZ_OK;
  }
  if (r >= (1ull << T.dev.k)) {
    *out = (uint32_t)e;
    return COLLATZ_OK;
  }
  if (!T.residues.empty()) {
    *out = (uint32_t)(std::lower_bound(T.residues.begin() + b, T.residues.begin() + e, r) - T.residues.begin());
    return COLLATZ_OK;
  }
  uint64_t lo = b, hi = e;  // binary search with single-entry reads
  while (lo < hi) {
    const uint64_t mid = (lo + hi) / 2;
    RangeEntry e;
    cudaError_t err = cudaMemcpy(&e, T.dev.table + mid, sizeof e, cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) return set_cuda_error(c, err, "lower_bound");
    const uint64_t rr = (uint64_t)e.r_lo | ((uint64_t)(e.meta & 0xFF) << 32);
    if (rr < r) lo = mid + 1; else hi = mid;
  }
  *out = (uint32_t)lo;
  return COLLATZ_OK;
}

int lower_range(collatz_ctx* c, const collatz_range& r, uint32_t req, const RangeTables& T,
                std::vector<RangeSeg>& segs, unsigned long long& items) {
  const uint32_t k = T.dev.k;
  const u128 O = u128_of(r.offset), S = r.size, E = O + S;
  if (r.size > (1ull << 48) || E > ((u128)1 << 96) || E < O) return COLLATZ_E_LIMIT;
  const uint32_t mod9 = (r.flags & COLLATZ_RANGE_NO_MOD9) ? 0u : 1u;
  // kept residues mod 9: {0,1,3,6,7} for T (cu:488), {0,2,3,6,8} for the negative variant
  const uint32_t keep9 = (r.flags & COLLATZ_RANGE_NEGATIVE) ? 0x14Du : 0xCBu;
  const u128 K = (u128)1 << k;
  if (S == 0) return COLLATZ_OK;
  if (O < K) {  // integers below 2^k: no residue sieve
    const uint64_t d_lo = (uint64_t)O, d_hi = (uint64_t)std::min(E, K);
    RangeSeg g{};
    g.item_begin = items;
    g.q_lo = d_lo;
    g.d_hi = d_hi;
    g.req = req;
    g.kind = 1;
    g.mod9 = mod9;
    segs.push_back(g);
    items += (d_hi - d_lo + DENSE_ITEM - 1) / DENSE_ITEM;
  }
  // Seeds >= 2^k: blocks q of 2^k residues.  The table is class-major (r mod
  // 9), and with the mod-9 sieve a block keeps exactly the classes c with
  // (q 2^k + c) mod 9 in {0,1,3,6,7}: 5 of the 9, depending only on q mod 9.
  // So each emitted segment covers one whole class (or, in a partial first
  // or last block, the class's residues in range), and every entry it names
  // is a seed.  Blocks strictly between the first and the last are grouped
  // by q mod 9 into segments with block stride 9.
  const u128 lo = std::max(O, K);
  if (lo >= E) return COLLATZ_OK;
  const u128 qa = lo >> k, qb = (E - 1) >> k;
  const uint32_t k9 = (uint32_t)(((u128)1 << (k % 6)) % 9);  // 2^k mod 9 (2^6 = 1 mod 9)
  auto live = [&](u128 q, uint32_t cl) {
    return !mod9 || ((keep9 >> (((uint32_t)(q % 9) * k9 + cl) % 9)) & 1u);
  };
  auto add = [&](u128 q, u128 nq, uint32_t stride, uint32_t s_lo, uint32_t s_hi) {
    if (s_lo >= s_hi || nq == 0) return;
    const uint32_t ipq = (s_hi - s_lo + RANGE_ITEM - 1) / RANGE_ITEM;
    const u128 max_nq = std::max<uint32_t>(1u, 0xFFFFFFFFu / ipq);  // < 2^32 items per segment
    while (nq > 0) {
      const uint32_t take = (uint32_t)std::min(nq, max_nq);
      RangeSeg g{};
      g.item_begin = items;
      g.q_lo = (uint64_t)q;
      g.q_hi = (uint32_t)(q >> 64);
      g.nq = take;
      g.s_lo = s_lo;
      g.s_hi = s_hi;
      g.ipq = ipq;
      g.req = req;
      g.kind = 0;
      g.qstride = (uint16_t)stride;
      g.mod9 = 0;  // every class of the segment is kept
      segs.push_back(g);
      items += (unsigned long long)take * ipq;
      q += (u128)take * stride;
      nq -= take;
    }
  };
  // one block q, residues [r0, r1)
  auto partial = [&](u128 q, uint64_t r0, uint64_t r1) -> int {
    for (uint32_t cl = 0; cl < 9; cl++) {
      if (!live(q, cl)) continue;
      uint32_t a = 0, b = 0;
      int rc = lower_bound_res(c, T, cl, r0, &a);
      if (!rc) rc = lower_bound_res(c, T, cl, r1, &b);
      if (rc) return rc;
      add(q, 1, 1, a, b);
    }
    return COLLATZ_OK;
  };
  const uint64_t ra = (uint64_t)(lo & (K - 1)), rb = (uint64_t)((E - 1) & (K - 1)) + 1;
  if (qa == qb) return partial(qa, ra, rb);
  int rc = partial(qa, ra, (uint64_t)K);
  if (rc) return rc;
  const u128 m0 = qa + 1, nm = qb - qa - 1;  // whole blocks in between
  if (nm > 0) {
    if (!mod9) {
      for (uint32_t cl = 0; cl < 9; cl++) add(m0, nm, 1, (uint32_t)T.dev.cls[cl], (uint32_t)T.dev.cls[cl + 1]);
    } else {
      for (uint32_t t = 0; t < 9 && (u128)t < nm; t++) {
        const u128 qt = m0 + t, nt = (nm - t + 8) / 9;  // blocks m0 + t, m0 + t + 9, ...
        for (uint32_t cl = 0; cl < 9; cl++)
          if (live(qt, cl)) add(qt, nt, 9, (uint32_t)T.dev.cls[cl], (uint32_t)T.dev.cls[cl + 1]);
      }
    }
  }
  return partial(qb, 0, rb);
}

}  // namespace cz

// =====================================================================
// Context.
// =====================================================================

extern "C" void collatz_config_default(collatz_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof *cfg);
  cfg->maxbits = 45;
  cfg->range_k = 24;
  cfg->device = 0;
  cfg->variant = COLLATZ_VARIANT_AUTO;
  cfg->iter_cap = 0;
}

extern "C" const char* collatz_status_string(int s) {
  switch (s) {
    case COLLATZ_OK: return "ok";
    case COLLATZ_E_ARG: return "invalid argument";
    case COLLATZ_E_CUDA: return "CUDA error";
    case COLLATZ_E_NOMEM: return "out of memory";
    case COLLATZ_E_LIMIT: return "request beyond limits";
    case COLLATZ_E_DEVICE: return "device reported an error";
    case COLLATZ_E_TIMEOUT: return "timed out";
    case COLLATZ_E_STATE: return "invalid state";
    case COLLATZ_E_ADMISSION: return "refused by device-memory admission";
    case COLLATZ_E_NODEV: return "no usable CUDA device";
    default: return "unknown status";
  }
}

extern "C" const char* collatz_last_error(const collatz_ctx* c) { return c ? c->err.c_str() : ""; }

extern "C" int collatz_create(const collatz_config* cfg, collatz_ctx** out) {
  if (!cfg || !out) return COLLATZ_E_ARG;
  *out = nullptr;
  if (cfg->maxbits < 16 || cfg->maxbits > 96) return COLLATZ_E_ARG;
  if (cfg->range_k < 8 || cfg->range_k > 34) return COLLATZ_E_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return COLLATZ_E_NODEV;
  }
  if (cfg->device < 0 || cfg->device >= ndev) return COLLATZ_E_ARG;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess) return COLLATZ_E_NODEV;
  if (prop.major != 10 || prop.minor != 0) return COLLATZ_E_NODEV;  // kernels are built for sm_100a only
  collatz_ctx* c = new collatz_ctx();
  c->cfg = *cfg;
  c->device = cfg->device;
  c->sm_count = prop.multiProcessorCount;
  int clk = 0;
  cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, c->device);
  c->sm_clock_khz = clk;
  if (cfg->iter_cap) c->iter_cap = cfg->iter_cap;
  if (cfg->variant != COLLATZ_VARIANT_AUTO) {
    if ((int)cfg->variant >= range_variants()) {
      delete c;
      return COLLATZ_E_ARG;
    }
    c->range_variant = (int)cfg->variant;
  }
  int rc = COLLATZ_OK;
  DeviceScope dev_scope(c->device);
  cudaError_t e = dev_scope.err;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
  for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaEventCreate(&c->ev[i]);
  if (e == cudaSuccess) e = range_init();
  if (e == cudaSuccess) e = range64_init();
  if (e == cudaSuccess) e = build_case_tables(&c->ct, cfg->maxbits, c->own_stream);
  if (e != cudaSuccess) {
    rc = set_cuda_error(c, e, "collatz_create");
    collatz_destroy(c);
    return rc;
  }
  c->stream = c->own_stream;
  if (cfg->variant == COLLATZ_VARIANT_AUTO) tune_on_create(c);
  *out = c;
  return COLLATZ_OK;
}

extern "C" void collatz_destroy(collatz_ctx* c) {
  if (!c) return;
  DeviceScope dev_scope(c->device);
  if (c->own_stream) cudaStreamSynchronize(c->own_stream);
  if (c->stream && c->stream != c->own_stream) cudaStreamSynchronize(c->stream);
  free_case_tables(&c->ct);
  for (auto& kv : c->rt) free_range_table(&kv.second.dev);
  DevBuf* bufs[] = {&c->d_rec, &c->d_counter, &c->d_overflow, &c->d_ovcount, &c->d_pairs[0], &c->d_pairs[1],
                    &c->d_segs, &c->d_widen, &c->d_widen2, &c->d_wcount, &c->t_seeds, &c->t_st, &c->t_exc,
                    &c->t_status, &c->t_idx[0], &c->t_idx[1], &c->t_cnt, &c->s1_front[0], &c->s1_front[1],
                    &c->s1_off, &c->s1_cnt, &c->s1_scal, &c->s1_stk_num, &c->s1_stk_meta, &c->s1_hist, &c->d_recs,
                    &c->d_rcursor, &c->d_first};
  for (DevBuf* b : bufs) b->release();
  c->h_rec.release();
  c->h_pairs.release();
  c->h_s1.release();
  c->h_segs.release();
  c->h_recs.release();
  for (auto& ev : c->ev)
    if (ev) cudaEventDestroy(ev);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

extern "C" int collatz_set_stream(collatz_ctx* c, void* s) {
  if (!c) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  c->stream = s ? (cudaStream_t)s : c->own_stream;
  return COLLATZ_OK;
}

extern "C" int collatz_device_info(const collatz_ctx* c, int* sm_count, int* sm_clock_khz) {
  if (!c) return COLLATZ_E_ARG;
  if (sm_count) *sm_count = c->sm_count;
  if (sm_clock_khz) *sm_clock_khz = c->sm_clock_khz;
  return COLLATZ_OK;
}

extern "C" int collatz_variant_count(int mode) {
  switch (mode) {
    case COLLATZ_MODE_CASES: return cases_variants();
    case COLLATZ_MODE_RANGE: return range_variants();
    case COLLATZ_MODE_RANGE64: return range64_variants();
    case COLLATZ_MODE_RANGE64_BITS: return (int)range64_max_seed_bits() + 1;
    default: return 0;
  }
}

extern "C" int collatz_set_variant(collatz_ctx* c, int mode, int v) {
  if (!c || v < 0 || v >= collatz_variant_count(mode)) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  switch (mode) {
    case COLLATZ_MODE_CASES: c->cases_variant = v; break;
    case COLLATZ_MODE_RANGE: c->range_variant = v; break;
    case COLLATZ_MODE_RANGE64: c->range64_variant = v; break;
    default: c->range64_bits = (uint32_t)v; break;
  }
  return COLLATZ_OK;
}

// =====================================================================
// Cases mode.
// =====================================================================

static int case_prepare(collatz_ctx* c) {
  CK(c, c->d_rec.ensure(sizeof(ReqRec)));
  CK(c, c->d_counter.ensure(sizeof(uint32_t) * 4));
  CK(c, c->d_overflow.ensure(sizeof(uint32_t) * 4 * OVERFLOW_CAP));
  CK(c, c->d_ovcount.ensure(sizeof(unsigned long long)));
  CK(c, c->h_rec.ensure(sizeof(ReqRec) + 64));
  CK(c, cudaMemsetAsync(c->d_rec.p, 0, sizeof(ReqRec), c->stream));
  CK(c, cudaMemsetAsync(c->d_ovcount.p, 0, sizeof(unsigned long long), c->stream));
  return COLLATZ_OK;
}

static CasesArgs case_args(collatz_ctx* c, const uint32_t* d_pairs, uint32_t npairs, int bigindex) {
  CasesArgs a;
  a.pairs = d_pairs;
  a.npairs = npairs;
  a.bigindex = bigindex;
  a.bv = c->ct.bv;
  a.mod9 = c->ct.mod9;
  a.magic = c->ct.magic;
  a.pow3 = c->ct.pow3;
  a.mbi = c->ct.mbi;
  a.tpo = c->ct.tpo;
  a.pair_counter = c->d_counter.as<uint32_t>();
  a.rec = c->d_rec.as<ReqRec>();
  a.overflow = c->d_overflow.as<uint32_t>();
  a.overflow_cap = OVERFLOW_CAP;
  a.overflow_count = c->d_ovcount.as<unsigned long long>();
  a.iter_cap = c->iter_cap;
  a.multi = 0;
  return a;
}

// Copies the record and the overflow list back (after the stream is idle).
static int case_finish(collatz_ctx* c, collatz_case_result* out) {
  ReqRec r;
  unsigned long long nov = 0;
  CK(c, cudaMemcpy(&r, c->d_rec.p, sizeof r, cudaMemcpyDeviceToHost));
  CK(c, cudaMemcpy(&nov, c->d_ovcount.p, sizeof nov, cudaMemcpyDeviceToHost));
  out->hash = r.hash;
  out->spot_checks = 0;
  out->seeds_checked = r.seeds;
  out->n_overflow = nov;
  out->errors = r.errors;
  if (r.valid & 2u) {
    std::memcpy(out->max_excursion, r.E, sizeof out->max_excursion);
    std::memcpy(out->max_excursion_seed, r.E_seed, sizeof out->max_excursion_seed);
  } else {
    std::memset(out->max_excursion, 0, sizeof out->max_excursion);
    std::memset(out->max_excursion_seed, 0, sizeof out->max_excursion_seed);
  }
  if (r.valid & 1u) {
    out->max_stopping_time = r.st;
    std::memcpy(out->max_stopping_time_seed, r.st_seed, sizeof out->max_stopping_time_seed);
  } else {
    out->max_stopping_time = 0;
    std::memset(out->max_stopping_time_seed, 0, sizeof out->max_stopping_time_seed);
  }
  const uint64_t have = std::min<uint64_t>(nov, OVERFLOW_CAP);
  if (out->overflow_seeds && out->overflow_cap && have) {
    std::vector<uint32_t> ov(4 * have);
    CK(c, cudaMemcpy(ov.data(), c->d_overflow.p, 16 * have, cudaMemcpyDeviceToHost));
    std::vector<u128> seeds(have);
    for (uint64_t i = 0; i < have; i++)
      seeds[i] = (u128)ov[4 * i] | ((u128)ov[4 * i + 1] << 32) | ((u128)ov[4 * i + 2] << 64);
    std::sort(seeds.begin(), seeds.end());
    const uint64_t n = std::min<uint64_t>(have, out->overflow_cap);
    for (uint64_t i = 0; i < n; i++) limbs4(seeds[i], out->overflow_seeds + 4 * i);
  }
  if (r.errors) {
    c->err = "device error bits " + hex_u32(r.errors);
    return COLLATZ_E_DEVICE;
  }
  return COLLATZ_OK;
}

extern "C" int collatz_verify_pairs(collatz_ctx* c, uint32_t bigindex, const uint32_t* pairs, uint32_t npairs,
                                    collatz_case_result* out) {
  if (!c || !out || (npairs && !pairs)) return COLLATZ_E_ARG;
  if (bigindex >= POW3_COUNT || (uint64_t)c->ct.tpo + bigindex >= POW3_COUNT) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  uint32_t* ovbuf = out->overflow_seeds;
  const uint64_t ovcap = out->overflow_cap;
  std::memset(out, 0, sizeof *out);
  out->overflow_seeds = ovbuf;
  out->overflow_cap = ovcap;
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  int rc = case_prepare(c);
  if (rc) return rc;
  if (npairs) {
    CK(c, c->d_pairs[0].ensure(32ull * npairs));
    CK(c, cudaMemcpyAsync(c->d_pairs[0].p, pairs, 32ull * npairs, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemsetAsync(c->d_counter.p, 0, sizeof(uint32_t), c->stream));
    CasesArgs a = case_args(c, c->d_pairs[0].as<uint32_t>(), npairs, (int)bigindex);
    CK(c, cudaEventRecord(c->ev[0], c->stream));
    CK(c, launch_cases(a, c->cases_variant, grid_for(c, 0, c->cases_variant), c->stream));
    CK(c, cudaEventRecord(c->ev[1], c->stream));
  }
  CK(c, cudaStreamSynchronize(c->stream));
  if (npairs) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    out->device_ms = ms;
    if (bigindex < 16) {
      out->pairs = npairs;
      out->launches = 1;  // launchkernel returns 1 for a non-empty batch (cu:648)
    } else {
      out->cpu_pairs = npairs;
    }
  }
  return case_finish(c, out);
}

extern "C" int collatz_step1_pairs(uint32_t maxbits, const collatz_case* cs, uint32_t* pairs, uint64_t cap,
                                   uint64_t* count) {
  if (!cs || !count || (cap && !pairs) || maxbits < 16 || maxbits > 96) return COLLATZ_E_ARG;
  const uint32_t mbi = maxbits - 10, tpo = mbi * 306 / 485 + 1;
  if (cs->sigfig > mbi || cs->threepower >= 128) return COLLATZ_E_ARG;
  Step1 s1(mbi, tpo);
  Step1Node root{u128_of(cs->base), cs->sigfig, cs->threepower, u128_of(cs->number), cs->doubleeven, cs->numevens};
  uint64_t n = 0;
  s1.leaves(root, [&](uint32_t bi, u128 b, u128 num) {
    if (n < cap) pack_pair(pairs + 8 * n, b, num, bi);
    n++;
  });
  *count = n;
  return COLLATZ_OK;
}

// The reference's counters from the leaves per bigindex (counts[16]: bigindex
// >= 16, the CPU path of cu:517-519): one launch per full bucket of 2^16
// pairs plus one per non-empty final flush (cu:532-534, 177-179).
static void leaf_counts_to_result(const uint64_t counts[17], collatz_case_result* out) {
  for (int b = 0; b < 16; b++) {
    out->pairs += counts[b];
    out->launches += (counts[b] + (1u << 16) - 1) >> 16;
  }
  out->cpu_pairs = counts[16];
}

extern "C" int collatz_step1_split(uint32_t maxbits, const collatz_case* cs, uint32_t cut, collatz_case* out,
                                   uint64_t cap, uint64_t* count) {
  if (!cs || !count || (cap && !out) || maxbits < 16 || maxbits > 96) return COLLATZ_E_ARG;
  const uint32_t mbi = maxbits - 10, tpo = mbi * 306 / 485 + 1;
  if (cs->sigfig > cut || cut > mbi || cs->threepower >= 128) return COLLATZ_E_ARG;
  Step1 s1(mbi, tpo);
  const Step1Node root{u128_of(cs->base), cs->sigfig, cs->threepower, u128_of(cs->number), cs->doubleeven,
                       cs->numevens};
  std::vector<Step1Node> nodes;
  s1.split(root, cut, nodes);
  *count = nodes.size();
  for (uint64_t i = 0; i < nodes.size() && i < cap; i++) {
    const Step1Node& r = nodes[i];
    out[i] = collatz_case{{(uint64_t)r.base, (uint64_t)(r.base >> 64)}, r.sigfig, r.threepower,
                          {(uint64_t)r.number, (uint64_t)(r.number >> 64)}, r.doubleeven, r.numevens};
  }
  return COLLATZ_OK;
}

namespace {

// Host Step 1 on all cores feeding batches of pairs to the GPU.
struct CasePipeline {
  std::mutex mu;
  std::condition_variable cv_free, cv_full;
  std::deque<int> free_bufs;
  std::deque<std::pair<int, uint32_t>> full;
  int workers_left = 0;
  uint32_t* host = nullptr;  // nbuf x CASE_BATCH pairs (pinned)

  int acquire() {
    std::unique_lock<std::mutex> l(mu);
    cv_free.wait(l, [&] { return !free_bufs.empty(); });
    const int b = free_bufs.front();
    free_bufs.pop_front();
    return b;
  }
  void submit(int b, uint32_t n) {
    {
      std::lock_guard<std::mutex> l(mu);
      full.emplace_back(b, n);
    }
    cv_full.notify_one();
  }
  void release(int b) {
    {
      std::lock_guard<std::mutex> l(mu);
      free_bufs.push_back(b);
    }
    cv_free.notify_one();
  }
};

struct CaseWorker {
  CasePipeline* P;
  int buf = -1;
  uint32_t n = 0;
  uint64_t counts[17] = {};  // [16] = bigindex >= 16
  static void leaf(void* vctx, uint32_t bi, u128 base, u128 number) {
    CaseWorker* w = (CaseWorker*)vctx;
    if (w->buf < 0) w->buf = w->P->acquire();
    pack_pair(w->P->host + (size_t)w->buf * CASE_BATCH * 8 + 8ull * w->n, base, number, bi);
    w->counts[bi < 16 ? bi : 16]++;
    if (++w->n == CASE_BATCH) {
      w->P->submit(w->buf, w->n);
      w->buf = -1;
      w->n = 0;
    }
  }
};

}  // namespace

// Step 1 on the host threads, batches copied to the device (the pipeline
// above); COLLATZ_CFG_HOST_STEP1.
static int run_case_host(collatz_ctx* c, const collatz_case* cs, collatz_case_result* out) {
  Step1 s1(c->ct.mbi, c->ct.tpo);
  const Step1Node root{u128_of(cs->base), cs->sigfig, cs->threepower, u128_of(cs->number), cs->doubleeven,
                       cs->numevens};
  unsigned hw = std::thread::hardware_concurrency();
  const int nthreads = (int)std::max(1u, std::min(hw ? hw : 1u, 64u));
  // split the tree until there are enough independent subtrees
  std::vector<Step1Node> roots;
  uint32_t cut = cs->sigfig;
  for (;;) {
    roots.clear();
    s1.split(root, cut, roots);
    if (roots.size() >= (size_t)8 * nthreads || cut >= c->ct.mbi) break;
    cut = std::min(c->ct.mbi, cut + 2);
  }

  const int nbuf = 2 * nthreads + 4;
  CK(c, c->h_pairs.ensure((size_t)nbuf * CASE_BATCH * 32));
  CK(c, c->d_pairs[0].ensure((size_t)CASE_BATCH * 32));
  CK(c, c->d_pairs[1].ensure((size_t)CASE_BATCH * 32));
  CasePipeline P;
  P.host = c->h_pairs.as<uint32_t>();
  for (int i = 0; i < nbuf; i++) P.free_bufs.push_back(i);
  P.workers_left = nthreads;
  std::atomic<size_t> next_root{0};
  std::vector<CaseWorker> ws(nthreads);
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; t++) {
    ws[t].P = &P;
    th.emplace_back([&, t] {
      CaseWorker& w = ws[t];
      for (;;) {
        const size_t i = next_root.fetch_add(1);
        if (i >= roots.size()) break;
        s1.leaves_fn(roots[i], &CaseWorker::leaf, &w);
      }
      if (w.buf >= 0 && w.n) P.submit(w.buf, w.n);
      else if (w.buf >= 0) P.release(w.buf);
      {
        std::lock_guard<std::mutex> l(P.mu);
        P.workers_left--;
      }
      P.cv_full.notify_one();
    });
  }

  // consumer: H2D on the copy stream, kernel on the compute stream
  cudaEvent_t copied[2], kdone[2];
  for (int i = 0; i < 2; i++) {
    cudaEventCreateWithFlags(&copied[i], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&kdone[i], cudaEventDisableTiming);
  }
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timing;
  uint64_t batches = 0;
  cudaError_t err = cudaSuccess;
  for (;;) {
    std::pair<int, uint32_t> job;
    {
      std::unique_lock<std::mutex> l(P.mu);
      P.cv_full.wait(l, [&] { return !P.full.empty() || P.workers_left == 0; });
      if (P.full.empty()) break;
      job = P.full.front();
      P.full.pop_front();
    }
    const int slot = (int)(batches & 1);
    if (err == cudaSuccess) {
      if (batches >= 2) err = cudaStreamWaitEvent(c->copy_stream, kdone[slot], 0);
      if (!err)
        err = cudaMemcpyAsync(c->d_pairs[slot].p, P.host + (size_t)job.first * CASE_BATCH * 8, 32ull * job.second,
                              cudaMemcpyHostToDevice, c->copy_stream);
      if (!err) err = cudaEventRecord(copied[slot], c->copy_stream);
      if (!err) err = cudaStreamWaitEvent(c->stream, copied[slot], 0);
      if (!err) err = cudaMemsetAsync(c->d_counter.p, 0, sizeof(uint32_t), c->stream);
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      timing.emplace_back(e0, e1);
      if (!err) err = cudaEventRecord(e0, c->stream);
      if (!err) {
        CasesArgs a = case_args(c, c->d_pairs[slot].as<uint32_t>(), job.second, -1);
        err = launch_cases(a, c->cases_variant, grid_for(c, 0, c->cases_variant), c->stream);
      }
      if (!err) err = cudaEventRecord(e1, c->stream);
      if (!err) err = cudaEventRecord(kdone[slot], c->stream);
      if (!err) err = cudaEventSynchronize(copied[slot]);
    }
    P.release(job.first);
    batches++;
  }
  for (auto& t : th) t.join();
  if (err == cudaSuccess) err = cudaStreamSynchronize(c->stream);
  double ms = 0;
  for (auto& ev : timing) {
    float x = 0;
    if (err == cudaSuccess) cudaEventElapsedTime(&x, ev.first, ev.second);
    ms += x;
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  for (int i = 0; i < 2; i++) {
    cudaEventDestroy(copied[i]);
    cudaEventDestroy(kdone[i]);
  }
  if (err != cudaSuccess) return set_cuda_error(c, err, "collatz_run_case");
  uint64_t counts[17] = {};
  for (auto& w : ws)
    for (int i = 0; i < 17; i++) counts[i] += w.counts[i];
  leaf_counts_to_result(counts, out);
  out->device_ms = ms;
  return case_finish(c, out);
}

// ---------------------------------------------------------------------
// Step 1 on the device (step1_dev.cu).
// ---------------------------------------------------------------------

namespace {

constexpr uint32_t S1_ROOTS = 2048;               // subtree roots cut on the host
constexpr uint64_t S1_FRONTIER_CAP = 1ull << 21;  // nodes of the last breadth-first level
constexpr uint64_t S1_CHUNK = 1ull << 22;         // pairs per emit pass and cases launch

struct S1Run {
  uint32_t nroots = 0, levels = 0, s0 = 0;
  const S1Node* front = nullptr;
  const uint32_t* front_count = nullptr;
  uint64_t total = 0;
  uint64_t hist[17] = {};
  float ms = 0;  // device time of the breadth-first levels and the count pass
};

Step1Args s1_args(collatz_ctx* c) {
  Step1Args a;
  std::memset(&a, 0, sizeof a);
  S1Scalars* sc = c->s1_scal.as<S1Scalars>();
  a.mbi = c->ct.mbi;
  a.tpo = c->ct.tpo;
  a.off = c->s1_off.as<unsigned long long>();
  a.cnt = c->s1_cnt.as<unsigned long long>();
  a.total = &sc->total;
  a.hist = sc->hist;
  a.stk_num = c->s1_stk_num.as<ulonglong2>();
  a.stk_meta = c->s1_stk_meta.as<uint4>();
  a.nthreads = (uint32_t)c->sm_count * STEP1_WALK_BLOCKS_PER_SM * 128u;
  return a;
}

}  // namespace

// Step 1 down to the leaf count of every frontier node, from the given roots
// (sigfig of each >= min_sig): the device expands as many breadth-first
// levels as the frontier buffer bounds (each level at most doubles), then
// the count pass walks every frontier node's subtree.  hist_lines (device,
// 17 counters per line, zeroed) receives the leaves per (line, bigindex) of a
// line batch; null for one case.  Ends with the stream idle.
static int s1_count_roots(collatz_ctx* c, const std::vector<S1Node>& roots, uint32_t min_sig,
                          unsigned long long* hist_lines, S1Run& R) {
  const uint32_t mbi = c->ct.mbi;
  R.nroots = (uint32_t)roots.size();
  if (roots.empty()) return COLLATZ_OK;
  if (roots.size() > S1_FRONTIER_CAP) return COLLATZ_E_LIMIT;
  uint64_t bound = R.nroots;
  uint32_t d = 0;
  while (min_sig + d < mbi && bound * 2 <= S1_FRONTIER_CAP) {
    bound *= 2;
    d++;
  }
  R.levels = d;
  R.s0 = min_sig + d;
  Step1Args a = s1_args(c);
  const uint64_t depth = mbi - R.s0;
  CK(c, c->s1_front[0].ensure(sizeof(S1Node) * bound));
  CK(c, c->s1_front[1].ensure(sizeof(S1Node) * bound));
  CK(c, c->s1_off.ensure(8 * bound));
  CK(c, c->s1_cnt.ensure(8 * bound));
  CK(c, c->s1_scal.ensure(sizeof(S1Scalars)));
  if (depth) {
    CK(c, c->s1_stk_num.ensure(16 * depth * a.nthreads));
    CK(c, c->s1_stk_meta.ensure(16 * depth * a.nthreads));
  }
  CK(c, c->h_s1.ensure(std::max(sizeof(S1Scalars), sizeof(S1Node) * (size_t)R.nroots + 4)));
  a = s1_args(c);  // buffers may have moved
  a.hist_lines = hist_lines;
  S1Node* hn = c->h_s1.as<S1Node>();
  std::memcpy(hn, roots.data(), sizeof(S1Node) * R.nroots);
  uint32_t* hcount = reinterpret_cast<uint32_t*>(hn + R.nroots);
  *hcount = R.nroots;
  S1Scalars* sc = c->s1_scal.as<S1Scalars>();
  CK(c, cudaEventRecord(c->ev[2], c->stream));
  CK(c, cudaMemsetAsync(sc, 0, sizeof(S1Scalars), c->stream));
  CK(c, cudaMemcpyAsync(c->s1_front[0].p, hn, sizeof(S1Node) * R.nroots, cudaMemcpyHostToDevice, c->stream));
  CK(c, cudaMemcpyAsync(&sc->level[0], hcount, 4, cudaMemcpyHostToDevice, c->stream));
  for (uint32_t l = 0; l < d; l++) {
    a.in = c->s1_front[l & 1].as<S1Node>();
    a.in_count = &sc->level[l];
    a.out = c->s1_front[(l + 1) & 1].as<S1Node>();
    a.out_count = &sc->level[l + 1];
    CK(c, launch_step1_expand(a, (uint32_t)((uint64_t)R.nroots << l), c->stream));
  }
  R.front = c->s1_front[d & 1].as<S1Node>();
  R.front_count = &sc->level[d];
  a.in = R.front;
  a.in_count = R.front_count;
  a.cursor = &sc->cursor[0];
  CK(c, launch_step1_walk(a, false, c->stream));
  CK(c, cudaEventRecord(c->ev[3], c->stream));
  S1Scalars* hs = c->h_s1.as<S1Scalars>();
  CK(c, cudaMemcpyAsync(&hs->total, &sc->total, 8 * 18, cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  R.total = hs->total;
  std::memcpy(R.hist, hs->hist, sizeof R.hist);
  CK(c, cudaEventElapsedTime(&R.ms, c->ev[2], c->ev[3]));
  return COLLATZ_OK;
}

// One case: the host cuts the tree at the first level with >= S1_ROOTS nodes
// (or at the leaves), then s1_count_roots.
static int s1_count(collatz_ctx* c, const collatz_case* cs, S1Run& R) {
  const uint32_t mbi = c->ct.mbi;
  Step1 s1(mbi, c->ct.tpo);
  const Step1Node root{u128_of(cs->base), cs->sigfig, cs->threepower, u128_of(cs->number), cs->doubleeven,
                       cs->numevens};
  std::vector<Step1Node> cut_nodes;
  uint32_t cut = cs->sigfig;
  for (;;) {
    cut_nodes.clear();
    s1.split(root, cut, cut_nodes);
    if (cut_nodes.size() >= S1_ROOTS || cut_nodes.empty() || cut >= mbi) break;
    cut++;
  }
  std::vector<S1Node> roots(cut_nodes.size());
  for (size_t i = 0; i < cut_nodes.size(); i++) {
    const Step1Node& r = cut_nodes[i];
    roots[i] = S1Node{(unsigned long long)r.base, (unsigned long long)(r.base >> 64), (unsigned long long)r.number,
                      (unsigned long long)(r.number >> 64), r.sigfig, r.threepower, r.doubleeven, r.numevens};
  }
  return s1_count_roots(c, roots, cut, nullptr, R);
}

// Emit pass: the pairs with leaf index in [lo, hi) to dst (device).
static cudaError_t s1_emit(collatz_ctx* c, const S1Run& R, uint64_t lo, uint64_t hi, uint32_t* dst) {
  Step1Args a = s1_args(c);
  S1Scalars* sc = c->s1_scal.as<S1Scalars>();
  a.in = R.front;
  a.in_count = R.front_count;
  a.cursor = &sc->cursor[1];
  a.pairs = dst;
  a.w_lo = lo;
  a.w_hi = hi;
  cudaError_t e = cudaMemsetAsync(a.cursor, 0, 4, c->stream);
  if (e == cudaSuccess) e = launch_step1_walk(a, true, c->stream);
  return e;
}

static int run_case_device(collatz_ctx* c, const collatz_case* cs, collatz_case_result* out) {
  S1Run R;
  int rc = s1_count(c, cs, R);
  if (rc) return rc;
  double ms = R.ms;
  if (R.total) {
    CK(c, c->d_pairs[0].ensure(32 * std::min<uint64_t>(R.total, S1_CHUNK)));
    uint32_t* dp = c->d_pairs[0].as<uint32_t>();
    CK(c, cudaEventRecord(c->ev[0], c->stream));
    for (uint64_t lo = 0; lo < R.total; lo += S1_CHUNK) {
      const uint64_t hi = std::min<uint64_t>(R.total, lo + S1_CHUNK);
      CK(c, s1_emit(c, R, lo, hi, dp));
      CK(c, cudaMemsetAsync(c->d_counter.p, 0, sizeof(uint32_t), c->stream));
      CasesArgs a = case_args(c, dp, (uint32_t)(hi - lo), -1);
      CK(c, launch_cases(a, c->cases_variant, grid_for(c, 0, c->cases_variant), c->stream));
    }
    CK(c, cudaEventRecord(c->ev[1], c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    float x = 0;
    CK(c, cudaEventElapsedTime(&x, c->ev[0], c->ev[1]));
    ms += x;
  }
  leaf_counts_to_result(R.hist, out);
  out->device_ms = ms;
  return case_finish(c, out);
}

extern "C" int collatz_run_case(collatz_ctx* c, const collatz_case* cs, collatz_case_result* out) {
  if (!c || !cs || !out) return COLLATZ_E_ARG;
  if (cs->sigfig > c->ct.mbi || cs->threepower >= 128) return COLLATZ_E_ARG;  // cu:515 is never reached
  std::lock_guard<std::recursive_mutex> g(c->mu);
  uint32_t* ovbuf = out->overflow_seeds;
  const uint64_t ovcap = out->overflow_cap;
  std::memset(out, 0, sizeof *out);
  out->overflow_seeds = ovbuf;
  out->overflow_cap = ovcap;
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  int rc = case_prepare(c);
  if (rc) return rc;
  return (c->cfg.flags & COLLATZ_CFG_HOST_STEP1) ? run_case_host(c, cs, out) : run_case_device(c, cs, out);
}

// Entry tests of search1 (cu:507-511) on a case's root, in the reference's
// 32-bit arithmetic.
static bool s1_root_pass(const collatz_case& cs) {
  if (485u * cs.threepower <= 306u * cs.sigfig) return false;
  if (cs.numevens >= 2u && cs.numevens % 2u == 0u && 306u * (cs.sigfig - 1u) >= 485u * (cs.threepower - 1u))
    return false;
  return true;
}

// Lines at least this many levels above the leaves (N-A - sigfig) run alone
// through the single-case path (host cut, one record): each has >= ~10^7
// seeds, enough to fill the GPU by itself, and the per-line records of a
// batch would only add work.  Shallower lines share batched passes.
constexpr uint32_t BATCH_ALONE_DEPTH = 20;

// One device pass over the lines cases[idx[0..m)] (line j of the pass is
// cases[idx[j]]); results go to out[idx[j]], overflow seeds to pool[used..).
static int batch_pass(collatz_ctx* c, const collatz_case* cases, const std::vector<uint32_t>& idx,
                      collatz_case_result* out, uint32_t* overflow_pool, uint64_t pool_cap, uint64_t& used) {
  const uint32_t n = (uint32_t)idx.size();
  int rc = case_prepare(c);
  if (rc) return rc;
  std::vector<S1Node> roots;
  uint32_t min_sig = 0xFFFFFFFFu;
  for (uint32_t i = 0; i < n; i++) {
    const collatz_case& cs = cases[idx[i]];
    if (!s1_root_pass(cs)) continue;  // search1 returns at once: no leaves
    roots.push_back(S1Node{cs.base[0], cs.base[1], cs.number[0], cs.number[1], cs.sigfig | (i << 8), cs.threepower,
                           cs.doubleeven, cs.numevens});
    min_sig = std::min(min_sig, cs.sigfig);
  }
  const size_t rb = sizeof(ReqRec) * n, hb = 17 * sizeof(unsigned long long) * n;
  CK(c, c->d_recs.ensure(rb));
  CK(c, c->s1_hist.ensure(hb));
  CK(c, cudaMemsetAsync(c->d_recs.p, 0, rb, c->stream));
  CK(c, cudaMemsetAsync(c->s1_hist.p, 0, hb, c->stream));
  S1Run R;
  rc = s1_count_roots(c, roots, min_sig, c->s1_hist.as<unsigned long long>(), R);
  if (rc) return rc;
  double ms = R.ms;
  if (R.total) {
    CK(c, c->d_pairs[0].ensure(32 * std::min<uint64_t>(R.total, S1_CHUNK)));
    uint32_t* dp = c->d_pairs[0].as<uint32_t>();
    CK(c, cudaEventRecord(c->ev[0], c->stream));
    for (uint64_t lo = 0; lo < R.total; lo += S1_CHUNK) {
      const uint64_t hi = std::min<uint64_t>(R.total, lo + S1_CHUNK);
      CK(c, s1_emit(c, R, lo, hi, dp));
      CK(c, cudaMemsetAsync(c->d_counter.p, 0, sizeof(uint32_t), c->stream));
      CasesArgs a = case_args(c, dp, (uint32_t)(hi - lo), -1);
      a.rec = c->d_recs.as<ReqRec>();
      a.multi = 1;
      int bps = 0;
      if (cases_occupancy(c->cases_variant, &bps, true) != cudaSuccess || bps <= 0) bps = 1;
      CK(c, launch_cases(a, c->cases_variant, (uint32_t)(bps * c->sm_count), c->stream));
    }
    CK(c, cudaEventRecord(c->ev[1], c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    float x = 0;
    CK(c, cudaEventElapsedTime(&x, c->ev[0], c->ev[1]));
    ms += x;
  }
  std::vector<ReqRec> recs(n);
  std::vector<uint64_t> hist(17ull * n);
  unsigned long long nov = 0;
  CK(c, cudaMemcpy(recs.data(), c->d_recs.p, rb, cudaMemcpyDeviceToHost));
  CK(c, cudaMemcpy(hist.data(), c->s1_hist.p, hb, cudaMemcpyDeviceToHost));
  CK(c, cudaMemcpy(&nov, c->d_ovcount.p, sizeof nov, cudaMemcpyDeviceToHost));
  // overflow seeds (4 words: limbs 0..2, line), grouped by line, ascending
  const uint64_t have = std::min<uint64_t>(nov, OVERFLOW_CAP);
  std::vector<uint32_t> ov(4 * have);
  if (have) CK(c, cudaMemcpy(ov.data(), c->d_overflow.p, 16 * have, cudaMemcpyDeviceToHost));
  std::vector<std::pair<uint32_t, u128>> tagged(have);
  for (uint64_t i = 0; i < have; i++)
    tagged[i] = {ov[4 * i + 3], (u128)ov[4 * i] | ((u128)ov[4 * i + 1] << 32) | ((u128)ov[4 * i + 2] << 64)};
  std::sort(tagged.begin(), tagged.end());
  uint64_t total_seeds = 0;
  for (uint32_t i = 0; i < n; i++) total_seeds += recs[i].seeds;
  uint64_t t = 0;
  int status = COLLATZ_OK;
  for (uint32_t i = 0; i < n; i++) {
    collatz_case_result& o = out[idx[i]];
    const ReqRec& r = recs[i];
    leaf_counts_to_result(&hist[17ull * i], &o);
    o.hash = r.hash;
    o.seeds_checked = r.seeds;
    o.n_overflow = r.items_done;
    o.errors = r.errors;
    if (r.valid & 2u) {
      std::memcpy(o.max_excursion, r.E, sizeof o.max_excursion);
      std::memcpy(o.max_excursion_seed, r.E_seed, sizeof o.max_excursion_seed);
    }
    if (r.valid & 1u) {
      o.max_stopping_time = r.st;
      std::memcpy(o.max_stopping_time_seed, r.st_seed, sizeof o.max_stopping_time_seed);
    }
    o.device_ms = total_seeds ? ms * (double)r.seeds / (double)total_seeds : 0.0;
    const uint64_t first = t;
    while (t < have && tagged[t].first == i) t++;
    const uint64_t k = std::min<uint64_t>(t - first, pool_cap - used);
    if (k) {
      o.overflow_seeds = overflow_pool + 4 * used;
      o.overflow_cap = k;
      for (uint64_t j = 0; j < k; j++) limbs4(tagged[first + j].second, o.overflow_seeds + 4 * j);
      used += k;
    }
    if (r.errors) status = COLLATZ_E_DEVICE;
  }
  return status;
}

extern "C" int collatz_run_case_batch(collatz_ctx* c, const collatz_case* cases, uint32_t n,
                                      collatz_case_result* out, uint32_t* overflow_pool, uint64_t pool_cap) {
  if (!c || !n || !cases || !out || (pool_cap && !overflow_pool)) return COLLATZ_E_ARG;
  if (n > COLLATZ_CASE_BATCH_MAX) return COLLATZ_E_LIMIT;
  for (uint32_t i = 0; i < n; i++)
    if (cases[i].sigfig > c->ct.mbi || cases[i].threepower >= 128) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  std::memset(out, 0, sizeof(collatz_case_result) * n);
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  uint64_t used = 0;
  int status = COLLATZ_OK;
  std::vector<uint32_t> shallow;
  std::vector<uint32_t> tmp;
  for (uint32_t i = 0; i < n; i++) {
    if (c->ct.mbi - cases[i].sigfig < BATCH_ALONE_DEPTH || !s1_root_pass(cases[i])) {
      shallow.push_back(i);
      continue;
    }
    int rc = case_prepare(c);
    if (rc) return rc;
    tmp.resize(4ull * OVERFLOW_CAP);
    collatz_case_result r;
    std::memset(&r, 0, sizeof r);
    r.overflow_seeds = tmp.data();
    r.overflow_cap = OVERFLOW_CAP;
    rc = (c->cfg.flags & COLLATZ_CFG_HOST_STEP1) ? run_case_host(c, &cases[i], &r) : run_case_device(c, &cases[i], &r);
    if (rc && rc != COLLATZ_E_DEVICE) return rc;
    if (rc) status = rc;
    const uint64_t k = std::min<uint64_t>(std::min<uint64_t>(r.n_overflow, OVERFLOW_CAP), pool_cap - used);
    r.overflow_seeds = nullptr;
    r.overflow_cap = 0;
    if (k) {
      r.overflow_seeds = overflow_pool + 4 * used;
      r.overflow_cap = k;
      std::memcpy(r.overflow_seeds, tmp.data(), 16 * k);
      used += k;
    }
    out[i] = r;
  }
  if (!shallow.empty()) {
    const int rc = batch_pass(c, cases, shallow, out, overflow_pool, pool_cap, used);
    if (rc && rc != COLLATZ_E_DEVICE) return rc;
    if (rc) status = rc;
  }
  if (status) c->err = "device error bits in a line of the batch";
  return status;
}

extern "C" int collatz_step1_pairs_device(collatz_ctx* c, const collatz_case* cs, uint32_t* pairs, uint64_t cap,
                                          uint64_t* count) {
  if (!c || !cs || !count || (cap && !pairs)) return COLLATZ_E_ARG;
  if (cs->sigfig > c->ct.mbi || cs->threepower >= 128) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  S1Run R;
  int rc = s1_count(c, cs, R);
  if (rc) return rc;
  *count = R.total;
  const uint64_t want = std::min<uint64_t>(cap, R.total);
  if (want) CK(c, c->d_pairs[0].ensure(32 * std::min<uint64_t>(want, S1_CHUNK)));
  for (uint64_t lo = 0; lo < want; lo += S1_CHUNK) {
    const uint64_t hi = std::min<uint64_t>(want, lo + S1_CHUNK);
    CK(c, s1_emit(c, R, lo, hi, c->d_pairs[0].as<uint32_t>()));
    CK(c, cudaMemcpyAsync(pairs + 8 * lo, c->d_pairs[0].p, 32 * (hi - lo), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
  }
  return COLLATZ_OK;
}

// =====================================================================
// Range plans.
// =====================================================================

struct collatz_plan {
  collatz_ctx* c = nullptr;
  uint32_t n = 0;
  RangeTables* T = nullptr;
  std::vector<RangeSeg> segs;
  unsigned long long items = 0;
  DevBuf d_segs, d_recs, d_cursor, d_widen, d_widen2, d_wcount, d_stats, d_first;
  HostBuf h_recs;
  bool stats = false, negative = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  float last_ms = 0;
};

// Checks that a batch uses one sieve (k, sign), fetches (or builds) its
// tables and lowers every request into segments.
static int range_lower_batch(collatz_ctx* c, const collatz_range* r, uint32_t n, RangeTables** T, uint32_t* k_out,
                             bool* neg_out, std::vector<RangeSeg>& segs, unsigned long long& items,
                             uint32_t* seed_bits, std::vector<uint32_t>& first_seg) {
  const uint32_t k = r[0].k ? r[0].k : c->cfg.range_k;
  const bool neg = (r[0].flags & COLLATZ_RANGE_NEGATIVE) != 0;
  for (uint32_t i = 0; i < n; i++)  // one sieve (k, sign) per launch
    if ((r[i].k ? r[i].k : c->cfg.range_k) != k || ((r[i].flags & COLLATZ_RANGE_NEGATIVE) != 0) != neg)
      return COLLATZ_E_ARG;
  if (k < 8 || k > 34) return COLLATZ_E_ARG;
  int rc = get_range_tables(c, k, T, neg);
  if (rc) return rc;
  *seed_bits = 0;
  first_seg.assign(n, ~0u);
  for (uint32_t i = 0; i < n; i++) {
    const size_t before = segs.size();
    rc = lower_range(c, r[i], i, **T, segs, items);
    if (rc) return rc;
    if (segs.size() > before) first_seg[i] = (uint32_t)before;  // the scouts' item
    *seed_bits = std::max(*seed_bits, range_seed_bits(r[i]));
  }
  if (segs.empty()) {  // keep the kernel's segment search well-defined
    RangeSeg g{};
    g.kind = 1;
    segs.push_back(g);
  }
  *k_out = k;
  *neg_out = neg;
  return COLLATZ_OK;
}

// Device buffers of one range launch.
struct RangeBufs {
  RangeSeg* segs;
  uint32_t nsegs;
  unsigned long long items;
  ReqRec* recs;
  void* h_recs;  // pinned: the records come back here
  uint32_t n;
  unsigned long long* cursor;
  WidenEntry* widen;
  WidenEntry* widen2;
  uint32_t* wcount;  // 2 counters
  unsigned long long* stats;
  const uint32_t* first_seg;  // per request: its first segment (threshold scouts)
};

static RangeArgs range_args(collatz_ctx* c, const RangeTables& T, uint32_t k, bool neg, const RangeBufs& b,
                            uint32_t seed_bits) {
  RangeArgs a;
  a.seed_bits = seed_bits;
  a.table = T.dev.table;
  a.k = k;
  a.segs = b.segs;
  a.nsegs = b.nsegs;
  a.item_cursor = b.cursor;
  a.item_limit = b.items;
  a.recs = b.recs;
  a.widen = b.widen;
  a.widen_cap = WIDEN_CAP;
  a.widen_count = b.wcount;
  a.iter_cap = c->iter_cap;
  a.stats = b.stats;
  a.negative = neg ? 1u : 0u;
  return a;
}

cudaError_t cz::range_kernel_launch(collatz_ctx* c, const RangeArgs& a, bool stats, cudaStream_t s) {
  if (!a.negative && a.seed_bits && a.seed_bits <= std::min(c->range64_bits, range64_max_seed_bits())) {
    const int v = c->range64_variant;
    int& bps = c->occ_range64[v & 7];
    if (bps <= 0 && (range64_occupancy(v, &bps) != cudaSuccess || bps <= 0)) bps = 1;
    const uint32_t grid = (uint32_t)(bps * c->sm_count);
    return stats ? launch_range64_stats(a, v, grid, s) : launch_range64(a, v, grid, s);
  }
  const int v = c->range_variant;
  int& bps = c->occ_range[v & 7];
  if (bps <= 0 && (range_occupancy(v, &bps) != cudaSuccess || bps <= 0)) bps = 1;
  const uint32_t grid = (uint32_t)(bps * c->sm_count);
  return (stats && !a.negative) ? launch_range_stats(a, grid, s) : launch_range(a, v, grid, s);
}

// One range launch on stream s: record and counter reset, k_range, the
// 192- and 256-bit widening passes, the record copy-back.  Captured into a
// graph by plans; issued directly by collatz_verify_batch.
static cudaError_t range_enqueue(collatz_ctx* c, const RangeArgs& a, const RangeBufs& b, cudaStream_t s) {
  const size_t rb = sizeof(ReqRec) * std::max(1u, b.n);
  cudaError_t e = cudaMemsetAsync(b.recs, 0, rb, s);
  if (!e) e = cudaMemsetAsync(b.cursor, 0, sizeof(unsigned long long), s);
  if (!e) e = cudaMemsetAsync(b.wcount, 0, sizeof(uint32_t) * 2, s);
  if (!e && b.stats) e = cudaMemsetAsync(b.stats, 0, 16 * sizeof(unsigned long long), s);
  if (!e && b.first_seg) e = launch_range_scout(a, b.first_seg, b.n, s);
  if (!e) e = range_kernel_launch(c, a, b.stats != nullptr, s);
  if (!e)
    e = launch_range_wide(b.widen, b.wcount, WIDEN_CAP, 6, b.recs, b.widen2, WIDEN_CAP, b.wcount + 1, c->iter_cap, s,
                          a.negative != 0);
  if (!e)
    e = launch_range_wide(b.widen2, b.wcount + 1, WIDEN_CAP, 8, b.recs, nullptr, 0, nullptr, c->iter_cap, s,
                          a.negative != 0);
  if (!e) e = cudaMemcpyAsync(b.h_recs, b.recs, rb, cudaMemcpyDeviceToHost, s);
  return e;
}

static bool range_stats_requested() {
  const char* dbg = getenv("COLLATZ_RANGE_STATS");
  return dbg && dbg[0] == '1';
}

static int plan_build(collatz_ctx* c, const collatz_range* r, uint32_t n, collatz_plan* p) {
  uint32_t k = 0, seed_bits = 0;
  std::vector<uint32_t> first_seg;
  int rc = range_lower_batch(c, r, n, &p->T, &k, &p->negative, p->segs, p->items, &seed_bits, first_seg);
  if (rc) return rc;
  p->n = n;
  CK(c, p->d_segs.ensure(sizeof(RangeSeg) * p->segs.size()));
  CK(c, cudaMemcpy(p->d_segs.p, p->segs.data(), sizeof(RangeSeg) * p->segs.size(), cudaMemcpyHostToDevice));
  CK(c, p->d_first.ensure(sizeof(uint32_t) * n));
  CK(c, cudaMemcpy(p->d_first.p, first_seg.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
  CK(c, p->d_recs.ensure(sizeof(ReqRec) * std::max(1u, n)));
  CK(c, p->h_recs.ensure(sizeof(ReqRec) * std::max(1u, n)));
  CK(c, p->d_cursor.ensure(sizeof(unsigned long long)));
  CK(c, p->d_widen.ensure(sizeof(WidenEntry) * WIDEN_CAP));
  CK(c, p->d_widen2.ensure(sizeof(WidenEntry) * WIDEN_CAP));
  CK(c, p->d_wcount.ensure(sizeof(uint32_t) * 2));
  p->stats = range_stats_requested();
  if (p->stats) CK(c, p->d_stats.ensure(16 * sizeof(unsigned long long)));
  const RangeBufs b{p->d_segs.as<RangeSeg>(), (uint32_t)p->segs.size(), p->items, p->d_recs.as<ReqRec>(),
                    p->h_recs.p, n, p->d_cursor.as<unsigned long long>(), p->d_widen.as<WidenEntry>(),
                    p->d_widen2.as<WidenEntry>(), p->d_wcount.as<uint32_t>(),
                    p->stats ? p->d_stats.as<unsigned long long>() : nullptr, p->d_first.as<uint32_t>()};
  const RangeArgs a = range_args(c, *p->T, k, p->negative, b, seed_bits);
  cudaStream_t s = c->own_stream;
  CK(c, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const cudaError_t e = range_enqueue(c, a, b, s);
  const cudaError_t e2 = cudaStreamEndCapture(s, &p->graph);
  if (e) return set_cuda_error(c, e, "plan capture");
  if (e2) return set_cuda_error(c, e2, "cudaStreamEndCapture");
  CK(c, cudaGraphInstantiate(&p->exec, p->graph, 0));
  return COLLATZ_OK;
}

extern "C" int collatz_plan_create(collatz_ctx* c, const collatz_range* r, uint32_t n, collatz_plan** out) {
  if (!c || !r || !n || !out) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  collatz_plan* p = new collatz_plan();
  p->c = c;
  int rc = plan_build(c, r, n, p);
  if (rc) {
    collatz_plan_destroy(p);
    return rc;
  }
  *out = p;
  return COLLATZ_OK;
}

extern "C" int collatz_plan_launch(collatz_plan* p) {
  if (!p || !p->exec) return COLLATZ_E_ARG;
  collatz_ctx* c = p->c;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  CK(c, cudaEventRecord(c->ev[2], c->stream));
  CK(c, cudaGraphLaunch(p->exec, c->stream));
  CK(c, cudaEventRecord(c->ev[3], c->stream));
  return COLLATZ_OK;
}

extern "C" int collatz_plan_results(collatz_plan* p, collatz_range_result* out) {
  if (!p || !out) return COLLATZ_E_ARG;
  collatz_ctx* c = p->c;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  CK(c, cudaStreamSynchronize(c->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
  const ReqRec* h = p->h_recs.as<ReqRec>();
  int status = COLLATZ_OK;
  if (p->stats) {  // diagnostics (COLLATZ_RANGE_STATS=1)
    unsigned long long st8[16];
    CK(c, cudaMemcpy(st8, p->d_stats.p, sizeof st8, cudaMemcpyDeviceToHost));
    fprintf(stderr,
            "collatz range stats: run_pairs=%llu slow_e=%llu replays=%llu jumps=%llu pops=%llu expansions=%llu "
            "passes=%llu offers=%llu windows=%llu pairs_64bit=%llu warp_cycles: offers=%llu refill=%llu "
            "lanes=%llu (refill: wait=%llu stage=%llu thresholds=%llu)\n",
            st8[0], st8[1], st8[2], st8[3], st8[4], st8[5], st8[6], st8[7], st8[14], st8[15], st8[8], st8[9],
            st8[10], st8[11], st8[12], st8[13]);
  }
  for (uint32_t i = 0; i < p->n; i++) {
    rec_to_range_result(h[i], &out[i]);
    out[i].device_ms = ms;
    if (out[i].status) status = out[i].status;
  }
  return status;
}

extern "C" void collatz_plan_destroy(collatz_plan* p) {
  if (!p) return;
  DeviceScope dev_scope(p->c->device);
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->d_segs.release();
  p->d_recs.release();
  p->d_cursor.release();
  p->d_widen.release();
  p->d_widen2.release();
  p->d_wcount.release();
  p->d_stats.release();
  p->d_first.release();
  p->h_recs.release();
  delete p;
}

// One-shot batches run directly on the context's grow-only scratch: no
// allocation, graph capture or free per call (each of those costs about a
// millisecond of host time, and cudaFree synchronises the device).
extern "C" int collatz_verify_batch(collatz_ctx* c, const collatz_range* r, uint32_t n, collatz_range_result* out) {
  if (!c || !r || !n || !out) return COLLATZ_E_ARG;
  if (range_stats_requested()) {  // diagnostics go through a plan
    collatz_plan* p = nullptr;
    int rc = collatz_plan_create(c, r, n, &p);
    if (rc) return rc;
    rc = collatz_plan_launch(p);
    if (!rc) rc = collatz_plan_results(p, out);
    collatz_plan_destroy(p);
    return rc;
  }
  std::lock_guard<std::recursive_mutex> g(c->mu);
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  std::vector<RangeSeg>& segs = c->range_segs;
  segs.clear();
  unsigned long long items = 0;
  RangeTables* T = nullptr;
  uint32_t k = 0, seed_bits = 0;
  bool neg = false;
  std::vector<uint32_t> first_seg;
  int rc = range_lower_batch(c, r, n, &T, &k, &neg, segs, items, &seed_bits, first_seg);
  if (rc) return rc;
  const size_t sb = sizeof(RangeSeg) * segs.size(), rb = sizeof(ReqRec) * n, fb = sizeof(uint32_t) * n;
  CK(c, c->d_segs.ensure(sb));
  CK(c, c->d_first.ensure(fb));
  CK(c, c->h_segs.ensure(sb + fb));  // the segments, then the scouts' first segments
  CK(c, c->d_recs.ensure(rb));
  CK(c, c->h_recs.ensure(rb));
  CK(c, c->d_rcursor.ensure(sizeof(unsigned long long)));
  CK(c, c->d_widen.ensure(sizeof(WidenEntry) * WIDEN_CAP));
  CK(c, c->d_widen2.ensure(sizeof(WidenEntry) * WIDEN_CAP));
  CK(c, c->d_wcount.ensure(sizeof(uint32_t) * 2));
  std::memcpy(c->h_segs.p, segs.data(), sb);
  std::memcpy(static_cast<char*>(c->h_segs.p) + sb, first_seg.data(), fb);
  const RangeBufs b{c->d_segs.as<RangeSeg>(), (uint32_t)segs.size(), items, c->d_recs.as<ReqRec>(), c->h_recs.p, n,
                    c->d_rcursor.as<unsigned long long>(), c->d_widen.as<WidenEntry>(),
                    c->d_widen2.as<WidenEntry>(), c->d_wcount.as<uint32_t>(), nullptr, c->d_first.as<uint32_t>()};
  const RangeArgs a = range_args(c, *T, k, neg, b, seed_bits);
  CK(c, cudaMemcpyAsync(c->d_segs.p, c->h_segs.p, sb, cudaMemcpyHostToDevice, c->stream));
  CK(c, cudaMemcpyAsync(c->d_first.p, static_cast<char*>(c->h_segs.p) + sb, fb, cudaMemcpyHostToDevice, c->stream));
  CK(c, cudaEventRecord(c->ev[2], c->stream));
  CK(c, range_enqueue(c, a, b, c->stream));
  CK(c, cudaEventRecord(c->ev[3], c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
  const ReqRec* h = c->h_recs.as<ReqRec>();
  int status = COLLATZ_OK;
  for (uint32_t i = 0; i < n; i++) {
    rec_to_range_result(h[i], &out[i]);
    out[i].device_ms = ms;
    if (out[i].status) status = out[i].status;
  }
  return status;
}

extern "C" int collatz_verify_range(collatz_ctx* c, const collatz_range* r, collatz_range_result* out) {
  return collatz_verify_batch(c, r, 1, out);
}

// =====================================================================
// Trajectory queries.
// =====================================================================

extern "C" int collatz_trajectory(collatz_ctx* c, const uint32_t* seeds, uint32_t n, uint64_t* st, uint32_t* exc,
                                  uint32_t* status) {
  if (!c || (n && (!seeds || !st || !exc || !status))) return COLLATZ_E_ARG;
  if (n == 0) return COLLATZ_OK;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  // seed ids sorted by limb class, then one launch for every class
  uint32_t cnt[5] = {0, 0, 0, 0, 0};
  std::vector<uint8_t> cls(n);
  for (uint32_t i = 0; i < n; i++) cnt[cls[i] = (uint8_t)traj_class(seeds + 8ull * i)]++;
  TrajAllArgs a;
  a.cstart[0] = 0;
  for (int j = 0; j < 5; j++) a.cstart[j + 1] = a.cstart[j] + cnt[j];
  CK(c, c->h_pairs.ensure(4ull * n));
  uint32_t* idx = c->h_pairs.as<uint32_t>();
  uint32_t fill[5];
  for (int j = 0; j < 5; j++) fill[j] = a.cstart[j];
  for (uint32_t i = 0; i < n; i++) idx[fill[cls[i]]++] = i;
  CK(c, c->t_seeds.ensure(32ull * n));
  CK(c, c->t_st.ensure(8ull * n));
  CK(c, c->t_exc.ensure(64ull * n));
  CK(c, c->t_status.ensure(4ull * n));
  CK(c, c->t_idx[0].ensure(4ull * n));
  CK(c, c->t_cnt.ensure(16));
  CK(c, cudaMemcpyAsync(c->t_seeds.p, seeds, 32ull * n, cudaMemcpyHostToDevice, c->stream));
  CK(c, cudaMemcpyAsync(c->t_idx[0].p, idx, 4ull * n, cudaMemcpyHostToDevice, c->stream));
  CK(c, cudaMemsetAsync(c->t_cnt.p, 0, 16, c->stream));
  a.seeds = c->t_seeds.as<uint32_t>();
  a.index = c->t_idx[0].as<uint32_t>();
  a.st = c->t_st.as<unsigned long long>();
  a.exc = c->t_exc.as<uint32_t>();
  a.status = c->t_status.as<uint32_t>();
  a.cursor = c->t_cnt.as<uint32_t>();
  a.iter_cap = c->iter_cap;
  const uint32_t grid = std::min<uint32_t>((n + 127) / 128, (uint32_t)c->sm_count * 8);
  CK(c, launch_traj_all(a, grid, c->stream));
  CK(c, cudaMemcpyAsync(st, c->t_st.p, 8ull * n, cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaMemcpyAsync(exc, c->t_exc.p, 64ull * n, cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaMemcpyAsync(status, c->t_status.p, 4ull * n, cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  return COLLATZ_OK;
}

extern "C" int collatz_case_tables(collatz_ctx* c, uint32_t* bv, uint32_t* mod9) {
  if (!c || !bv || !mod9) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  CK(c, cudaMemcpy(bv, c->ct.bv, sizeof(uint32_t) * 16 * BV_WORDS_HOST, cudaMemcpyDeviceToHost));
  CK(c, cudaMemcpy(mod9, c->ct.mod9, sizeof(uint32_t) * 9 * 32, cudaMemcpyDeviceToHost));
  return COLLATZ_OK;
}

extern "C" int collatz_range_sieve(collatz_ctx* c, uint32_t k, uint8_t* bits, uint64_t* count) {
  if (!c || k < 8 || k > 34) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  DeviceScope dev_scope(c->device);
  CK(c, dev_scope.err);
  RangeTables* T = nullptr;
  int rc = get_range_tables(c, k, &T);
  if (rc) return rc;
  if (count) *count = T->dev.count;
  if (bits) CK(c, cudaMemcpy(bits, T->dev.bits, (1ull << k) / 8, cudaMemcpyDeviceToHost));
  return COLLATZ_OK;
}
