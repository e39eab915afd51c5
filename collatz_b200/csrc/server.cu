// server.cu -- serving mode: continuous batching of range verifications and
// trajectory queries on one device (collatz_server_* in include/collatz.h).
//
// The server owns a context (sieve tables resident in HBM), a budget thread
// (the admission budget's reads of free device memory, below) and two worker
// threads, each with its own stream:
//   range thread  -- slices.  A slice is one launch of the persistent range
//                    kernel over a work list cut from the admitted range
//                    requests of one sieve exponent k (water-filling: requests
//                    that need less than an equal share take what they need,
//                    the rest of the slice budget goes to the larger ones),
//                    followed by the 192- and 256-bit widening passes and a
//                    copy of the request records; a prologue kernel zeroes the
//                    slice's counters and the records of newly admitted
//                    requests.  Two slices are kept in
//                    flight, so the next one is queued behind the running one
//                    and the device does not wait for the host.  A request's
//                    record lives in one device slot for its whole life, so
//                    its maxima and counts accumulate over slices exactly as
//                    in a single launch.
//   query thread  -- trajectory batches (higher-priority stream).  Admitted
//                    queries are concatenated into one batch: seeds are sorted
//                    by bit length into limb classes on the host, and one
//                    launch serves every class (a seed that needs wider values
//                    is run again by its thread).  Two batches are kept in
//                    flight.  The host copies of a batch (gathering seeds,
//                    scattering results into the callers' buffers) run on this
//                    thread and a small pool of helpers, off the range path.
// Admission (arrival order within each kind) needs a free request slot and,
// for a query, free device memory: cudaMemGetInfo's free bytes plus this
// server's idle pool memory, minus the bytes promised to admitted queries
// that have not allocated yet, minus hbm_reserve.  A budget thread re-reads
// these every 50 ms (and when a query does not fit), so admission itself
// makes no CUDA call: cudaMemGetInfo has taken hundreds of milliseconds under
// load.  A query needs 128 bytes per seed; a range request needs its record
// slot only.  A request that could not fit
// even on an otherwise empty device is refused (COLLATZ_E_ADMISSION); one
// that does not fit now waits.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime.h"

using namespace cz;

namespace {

using Clock = std::chrono::steady_clock;

constexpr int SLICE_DEPTH = 2;  // range slices in flight
constexpr int BATCH_DEPTH = 2;  // trajectory batches in flight
constexpr uint64_t TRAJ_BYTES_PER_SEED = 128;
constexpr uint32_t MAX_ACTIVE_LIMIT = 4096;
constexpr uint32_t MAX_BATCH_SEEDS = 1u << 22;
// Staging reserved per admitted request for a slice's work list: a request
// lowers to a dense part, up to 5 class segments for each partial block and
// up to 45 (9 residues of q mod 9 x 5 kept classes) for the whole blocks in
// between; more is allocated on demand.
constexpr size_t SEGS_PER_REQ = 64;

// host-time buckets of the worker threads
enum { T_ADMIT, T_BUILD, T_COMPLETE, T_IDLE, T_N };

struct Req {
  uint64_t ticket = 0;
  collatz_request q{};
  int32_t status = COLLATZ_OK;
  double submit_s = 0, admit_s = 0, done_s = 0;
  // range requests
  uint32_t k = 0, slot = 0;
  bool neg = false;            // the negative-integer variant
  std::vector<RangeSeg> segs;  // lowered work list, item_begin relative to the request
  unsigned long long items = 0, cursor = 0;
  size_t seg_i = 0;            // segment holding the cursor
  collatz_range_result res{};
  // trajectory queries
  uint64_t dev_bytes = 0;
  uint32_t batch_off = 0;
};

struct Slice {
  DevBuf d_segs, d_cursor, d_widen[2], d_wcount;
  HostBuf h_segs, h_recs;
  std::vector<Req*> finishing;
  cudaEvent_t t0 = nullptr, done = nullptr;
  bool busy = false;
};

// Byte layout of a trajectory batch of n seeds in its device block:
//   [0, 32n) seeds (8 words each) | [32n, 36n) class lists | o_cnt: 16 cursor
//   words | o_out: stopping times (8n), excursions (64n), statuses (4n).
struct BatchLayout {
  uint64_t o_idx, o_cnt, in_bytes, o_out, r_st, r_exc, r_status, out_bytes;
  explicit BatchLayout(uint64_t n)
      : o_idx(32 * n), o_cnt((36 * n + 255) & ~255ull), in_bytes(o_cnt + 64), o_out(o_cnt + 256),
        r_st(0), r_exc(8 * n), r_status(72 * n), out_bytes(76 * n) {}
};

struct Batch {
  // h_in mirrors the input part of the batch's device block (seeds, class
  // lists, cursors) and h_out its output part (stopping times, excursions,
  // statuses), so that each direction is one copy
  HostBuf h_in, h_out;
  std::vector<Req*> reqs;
  std::vector<uint8_t> cls;
  uint32_t n = 0;
  cudaEvent_t done = nullptr;
  bool busy = false;
};

double since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

// A slice's prologue: zeroes its item cursor and widen counters and the
// records of the requests admitted since the previous slice (one launch in
// place of a memset per request).
__global__ void k_slice_prologue(unsigned long long* cursor, uint32_t* wcount, ReqRec* recs, const uint32_t* slots,
                                 uint32_t nslots) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    *cursor = 0;
    wcount[0] = 0;
    wcount[1] = 0;
  }
  constexpr uint32_t W = sizeof(ReqRec) / 8;  // 17 words of 8 bytes
  for (uint32_t i = t; i < nslots * W; i += gridDim.x * blockDim.x)
    reinterpret_cast<unsigned long long*>(recs + slots[i / W])[i % W] = 0ull;
}

// A fixed set of host threads for the query path's copies (gathering query
// seeds into the pinned batch, scattering results into the callers'
// buffers).  run(parts, fn) calls fn(p) for every p in [0, parts) on the pool
// and on the calling thread, and returns when all have finished.  One caller
// at a time (the query thread).
struct CopyPool {
  std::vector<std::thread> th;
  std::mutex mu;
  std::condition_variable cv, cv_done;
  std::function<void(int)> job;
  std::atomic<int> next{0}, done{0};
  int parts = 0;
  uint64_t gen = 0;
  bool stop = false;

  void work() {
    for (int p; (p = next.fetch_add(1)) < parts;) {
      job(p);
      if (done.fetch_add(1) + 1 == parts) {
        std::lock_guard<std::mutex> g(mu);
        cv_done.notify_all();
      }
    }
  }
  void start(int n) {
    for (int i = 0; i < n; i++)
      th.emplace_back([this] {
        uint64_t seen = 0;
        for (;;) {
          {
            std::unique_lock<std::mutex> g(mu);
            cv.wait(g, [&] { return stop || gen != seen; });
            if (stop) return;
            seen = gen;
          }
          work();
        }
      });
  }
  void run(int nparts, const std::function<void(int)>& fn) {
    if (nparts <= 1 || th.empty()) {
      for (int p = 0; p < nparts; p++) fn(p);
      return;
    }
    {
      std::lock_guard<std::mutex> g(mu);
      job = fn;
      parts = nparts;
      next = 0;
      done = 0;
      gen++;
    }
    cv.notify_all();
    work();
    std::unique_lock<std::mutex> g(mu);
    cv_done.wait(g, [&] { return done.load() >= parts; });
  }
  void shutdown() {
    {
      std::lock_guard<std::mutex> g(mu);
      stop = true;
    }
    cv.notify_all();
    for (std::thread& t : th) t.join();
    th.clear();
  }
};

constexpr uint64_t COPY_PART_SEEDS = 1u << 14;  // seeds per part of a parallel copy

}  // namespace

struct collatz_server {
  collatz_server_config cfg{};
  collatz_ctx* ctx = nullptr;
  cudaStream_t sa = nullptr, sb = nullptr;
  cudaMemPool_t pool = nullptr;
  Clock::time_point t0;
  size_t total_mem = 0;

  // guarded by mu
  std::mutex mu;
  std::condition_variable cv_range, cv_query, cv_done;
  std::deque<Req*> pend_range, pend_query;
  std::unordered_map<uint64_t, Req*> done;
  std::unordered_map<uint64_t, Req*> known;  // tickets not yet collected
  uint64_t next_ticket = 1;
  bool stopping = false;
  collatz_server_info_t info{};
  double host_t[2][T_N] = {};  // [range, query thread][bucket]

  std::atomic<uint32_t> active[2] = {{0}, {0}};  // admitted, not yet complete: [0] ranges, [1] queries

  // query admission budget (guarded by mb), re-read by the budget thread
  std::mutex mb;
  std::condition_variable cv_budget;
  int64_t budget = 0;
  uint64_t promised = 0;  // admitted query bytes not yet allocated
  uint64_t launched = 0;  // query bytes moved from promised to the pool, in total
  bool want_budget = false, budget_stop = false;
  std::thread thr_budget;

  // range thread only
  std::vector<Req*> ranges;  // admitted range requests not yet complete
  std::vector<uint32_t> free_slots;
  std::vector<uint32_t> fresh_slots;  // records of admitted requests, zeroed by the next slice's prologue
  DevBuf d_recs;
  Slice slices[SLICE_DEPTH];
  std::deque<int> slice_order;
  // query thread only
  std::deque<Req*> queries;  // admitted queries not yet in a batch
  Batch batches[BATCH_DEPTH];
  std::deque<int> batch_order;

  std::thread thr_range, thr_query;
  CopyPool copy_pool;
};

namespace {

void publish(collatz_server* s, Req* r, int status) {
  r->status = status;
  r->done_s = since(s->t0);
  std::lock_guard<std::mutex> g(s->mu);
  s->done[r->ticket] = r;
  s->info.completed++;
  if (status == COLLATZ_E_ADMISSION) s->info.refused++;
  s->cv_done.notify_all();
}

// Re-reads the device's free memory into the admission budget (called
// without mb held; the CUDA calls run outside it): free bytes plus this
// server's idle pool memory, minus the bytes promised to admitted queries
// that have not allocated yet, minus hbm_reserve, minus the bytes that
// reached the pool while the read ran (they may be missing from it).
// Between reads each admission takes its bytes from the budget and frees are
// not credited, so the budget never over-states what is free.
void refresh_budget(collatz_server* s) {
  uint64_t launched0 = 0;
  {
    std::lock_guard<std::mutex> g(s->mb);
    launched0 = s->launched;
  }
  size_t fr = 0, tot = 0;
  const bool ok = cudaMemGetInfo(&fr, &tot) == cudaSuccess;
  if (!ok) cudaGetLastError();
  uint64_t reserved = 0, used = 0;
  cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
  cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrUsedMemCurrent, &used);
  uint64_t promised = 0;
  {
    std::lock_guard<std::mutex> g(s->mb);
    promised = s->promised;
    s->budget = ok ? (int64_t)fr + (int64_t)(reserved - used) - (int64_t)promised -
                         (int64_t)(s->launched - launched0) - (int64_t)s->cfg.hbm_reserve
                   : -1;
  }
  std::lock_guard<std::mutex> g(s->mu);
  s->info.hbm_free = fr;
  s->info.hbm_admitted = promised + used;
}

// Budget thread: re-reads the budget every 50 ms, or at most every
// millisecond while a query waits for memory, and wakes the query thread.
void budget_loop(collatz_server* s) {
  cudaSetDevice(s->ctx->device);
  std::unique_lock<std::mutex> g(s->mb);
  while (!s->budget_stop) {
    s->cv_budget.wait_for(g, std::chrono::milliseconds(50), [s] { return s->want_budget || s->budget_stop; });
    if (s->budget_stop) break;
    s->want_budget = false;
    g.unlock();
    refresh_budget(s);
    s->cv_query.notify_one();
    std::this_thread::sleep_for(std::chrono::milliseconds(1));
    g.lock();
  }
}

// Takes need bytes from the budget if they fit; else asks the budget thread
// for a fresh read.
bool take_budget(collatz_server* s, uint64_t need) {
  std::lock_guard<std::mutex> g(s->mb);
  if (s->budget < (int64_t)need) {
    s->want_budget = true;
    s->cv_budget.notify_one();
    return false;
  }
  s->budget -= (int64_t)need;
  s->promised += need;
  return true;
}

// Each kind has its own max_active admissions, so a backlog of range
// requests never holds back trajectory queries (or the other way round).
bool take_active(collatz_server* s, int kind) {
  uint32_t a = s->active[kind].load();
  while (a < s->cfg.max_active)
    if (s->active[kind].compare_exchange_weak(a, a + 1)) return true;
  return false;
}

// Next queued request of one kind, or nullptr.  Requests that could not fit
// even on an otherwise empty device are refused on the way.
Req* front(collatz_server* s, std::deque<Req*>& q, uint64_t need_per_seed) {
  for (;;) {
    Req* r = nullptr;
    {
      std::lock_guard<std::mutex> g(s->mu);
      if (q.empty()) return nullptr;
      r = q.front();
      const uint64_t need = need_per_seed ? need_per_seed * r->q.nseeds + 256 : 0;
      if ((int64_t)s->total_mem - (int64_t)s->cfg.hbm_reserve >= (int64_t)need) return r;
      q.pop_front();
    }
    publish(s, r, COLLATZ_E_ADMISSION);
  }
}

void pop_admitted(collatz_server* s, std::deque<Req*>& q, Req* r) {
  r->admit_s = since(s->t0);
  std::lock_guard<std::mutex> g(s->mu);
  q.pop_front();
  s->info.admitted++;
}

// ---------------------------------------------------------------------
// range thread
// ---------------------------------------------------------------------

// Admits queued range requests in arrival order while request slots and
// memory allow, and lowers them (the survivor table of their k is built on
// first use and stays resident).
void admit_ranges(collatz_server* s) {
  collatz_ctx* c = s->ctx;
  for (;;) {
    Req* r = front(s, s->pend_range, 0);
    if (!r || s->free_slots.empty()) return;
    if (!take_active(s, 0)) return;
    pop_admitted(s, s->pend_range, r);
    r->k = r->q.range.k ? r->q.range.k : c->cfg.range_k;
    r->neg = (r->q.range.flags & COLLATZ_RANGE_NEGATIVE) != 0;
    RangeTables* T = nullptr;
    int rc = get_range_tables(c, r->k, &T, r->neg);
    if (!rc) rc = lower_range(c, r->q.range, 0, *T, r->segs, r->items);
    if (rc || r->items == 0) {  // an error, or no seed in the range
      s->active[0]--;
      publish(s, r, rc);
      continue;
    }
    // the record is zeroed by the prologue of the next slice, which runs before any slice
    // that holds this request (slices run in order on one stream)
    r->slot = s->free_slots.back();
    s->free_slots.pop_back();
    s->fresh_slots.push_back(r->slot);
    s->ranges.push_back(r);
  }
}

// Appends up to quota work items of r (from its cursor) to a slice.
void take_items(Req* r, unsigned long long quota, std::vector<RangeSeg>& out, unsigned long long& slice_items) {
  unsigned long long taken = 0;
  while (taken < quota && r->seg_i < r->segs.size()) {
    const RangeSeg& g = r->segs[r->seg_i];
    const unsigned long long g_items =
        ((r->seg_i + 1 < r->segs.size()) ? r->segs[r->seg_i + 1].item_begin : r->items) - g.item_begin;
    const unsigned long long local = r->cursor - g.item_begin;
    const unsigned long long n = std::min(g_items - local, quota - taken);
    RangeSeg p = g;
    p.item_begin = slice_items;
    p.local0_lo = (uint32_t)local;
    p.local0_hi = (uint32_t)(local >> 32);
    p.req = r->slot;
    out.push_back(p);
    slice_items += n;
    taken += n;
    r->cursor += n;
    if (local + n == g_items) r->seg_i++;
  }
}

// Builds and enqueues one range slice.  Returns 1 if one was launched, 0 if
// there is no range work, negative on error.
int launch_slice(collatz_server* s, int si) {
  // the sieve (exponent k, sign) of the oldest request with work left
  uint32_t k = 0;
  bool neg = false;
  uint64_t oldest = ~0ull;
  for (Req* r : s->ranges)
    if (r->cursor < r->items && r->ticket < oldest) {
      oldest = r->ticket;
      k = r->k;
      neg = r->neg;
    }
  if (!k) return 0;
  std::vector<std::pair<unsigned long long, Req*>> want;
  for (Req* r : s->ranges)
    if (r->cursor < r->items && r->k == k && r->neg == neg) want.push_back({r->items - r->cursor, r});
  std::sort(want.begin(), want.end(),
            [](const std::pair<unsigned long long, Req*>& a, const std::pair<unsigned long long, Req*>& b) {
              return a.first != b.first ? a.first < b.first : a.second->ticket < b.second->ticket;
            });
  Slice& S = s->slices[si];
  S.finishing.clear();
  std::vector<RangeSeg> segs;
  unsigned long long slice_items = 0, budget = s->cfg.slice_items;
  uint32_t seed_bits = 0;
  std::vector<uint32_t> scouts;  // the first segment of each request that starts in this slice
  for (size_t i = 0; i < want.size(); i++) {
    const unsigned long long share = std::max<unsigned long long>(1, budget / (want.size() - i));
    const unsigned long long q = std::min(want[i].first, share);
    if (q) seed_bits = std::max(seed_bits, range_seed_bits(want[i].second->q.range));
    const bool starts = want[i].second->cursor == 0;
    const size_t before = segs.size();
    take_items(want[i].second, q, segs, slice_items);
    if (starts && segs.size() > before) scouts.push_back((uint32_t)before);
    budget -= std::min(budget, q);
    if (want[i].second->cursor == want[i].second->items) S.finishing.push_back(want[i].second);
  }
  collatz_ctx* c = s->ctx;
  RangeTables* T = nullptr;
  int rc = get_range_tables(c, k, &T, neg);
  if (rc) return rc;
  const size_t sb = sizeof(RangeSeg) * segs.size(), fb = sizeof(uint32_t) * scouts.size();
  const size_t zb = sizeof(uint32_t) * s->fresh_slots.size();
  const size_t rb = sizeof(ReqRec) * s->cfg.max_active;
  // one upload: the segments, the scouts' segment indices, the records to zero
  cudaError_t e = S.d_segs.ensure(sb + fb + zb);
  if (!e) e = S.h_segs.ensure(sb + fb + zb);
  if (!e) e = S.h_recs.ensure(rb);
  if (e) return set_cuda_error(c, e, "server slice buffers");
  std::memcpy(S.h_segs.p, segs.data(), sb);
  if (fb) std::memcpy(static_cast<char*>(S.h_segs.p) + sb, scouts.data(), fb);
  if (zb) std::memcpy(static_cast<char*>(S.h_segs.p) + sb + fb, s->fresh_slots.data(), zb);
  const uint32_t nfresh = (uint32_t)s->fresh_slots.size();
  s->fresh_slots.clear();
  RangeArgs a;
  a.table = T->dev.table;
  a.k = k;
  a.segs = S.d_segs.as<RangeSeg>();
  a.nsegs = (uint32_t)segs.size();
  a.item_cursor = S.d_cursor.as<unsigned long long>();
  a.item_limit = slice_items;
  a.recs = s->d_recs.as<ReqRec>();
  a.widen = S.d_widen[0].as<WidenEntry>();
  a.widen_cap = WIDEN_CAP;
  a.widen_count = S.d_wcount.as<uint32_t>();
  a.iter_cap = c->iter_cap;
  a.stats = nullptr;
  a.negative = neg ? 1u : 0u;
  a.seed_bits = seed_bits;
  cudaStream_t st = s->sa;
  e = cudaMemcpyAsync(S.d_segs.p, S.h_segs.p, sb + fb + zb, cudaMemcpyHostToDevice, st);
  if (!e) {
    const uint32_t words = nfresh * (uint32_t)(sizeof(ReqRec) / 8);
    k_slice_prologue<<<std::max(1u, std::min(64u, (words + 255) / 256)), 256, 0, st>>>(
        S.d_cursor.as<unsigned long long>(), S.d_wcount.as<uint32_t>(), s->d_recs.as<ReqRec>(),
        reinterpret_cast<const uint32_t*>(static_cast<const char*>(S.d_segs.p) + sb + fb), nfresh);
    e = cudaGetLastError();
  }
  if (!e) e = cudaEventRecord(S.t0, st);
  // threshold scouts for the requests that start here (their records were zeroed by the prologue)
  if (!e && fb)
    e = launch_range_scout(a, reinterpret_cast<const uint32_t*>(static_cast<const char*>(S.d_segs.p) + sb),
                           (uint32_t)scouts.size(), st);
  if (!e) e = range_kernel_launch(c, a, false, st);
  if (!e)
    e = launch_range_wide(S.d_widen[0].as<WidenEntry>(), S.d_wcount.as<uint32_t>(), WIDEN_CAP, 6, a.recs,
                          S.d_widen[1].as<WidenEntry>(), WIDEN_CAP, S.d_wcount.as<uint32_t>() + 1, c->iter_cap, st,
                          neg);
  if (!e)
    e = launch_range_wide(S.d_widen[1].as<WidenEntry>(), S.d_wcount.as<uint32_t>() + 1, WIDEN_CAP, 8, a.recs,
                          nullptr, 0, nullptr, c->iter_cap, st, neg);
  if (!e && !S.finishing.empty()) e = cudaMemcpyAsync(S.h_recs.p, s->d_recs.p, rb, cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaEventRecord(S.done, st);
  if (e) return set_cuda_error(c, e, "server slice launch");
  S.busy = true;
  s->slice_order.push_back(si);
  std::lock_guard<std::mutex> g(s->mu);
  s->info.range_slices++;
  return 1;
}

void complete_slice(collatz_server* s, int si) {
  Slice& S = s->slices[si];
  float ms = 0;
  cudaEventElapsedTime(&ms, S.t0, S.done);
  const ReqRec* recs = S.h_recs.as<ReqRec>();
  uint64_t seeds = 0;
  for (Req* r : S.finishing) {
    rec_to_range_result(recs[r->slot], &r->res);
    seeds += r->res.seeds_checked;
    s->free_slots.push_back(r->slot);
    s->ranges.erase(std::find(s->ranges.begin(), s->ranges.end(), r));
    s->active[0]--;
    publish(s, r, r->res.status);
  }
  S.busy = false;
  std::lock_guard<std::mutex> g(s->mu);
  s->info.device_busy_s += ms / 1e3;
  s->info.range_seeds_checked += seeds;
}

// ---------------------------------------------------------------------
// query thread
// ---------------------------------------------------------------------

void admit_queries(collatz_server* s) {
  for (;;) {
    Req* r = front(s, s->pend_query, TRAJ_BYTES_PER_SEED);
    if (!r) return;
    const uint64_t need = TRAJ_BYTES_PER_SEED * r->q.nseeds + 768;  // covers BatchLayout's padding
    if (!take_active(s, 1)) return;
    if (!take_budget(s, need)) {
      s->active[1]--;
      return;
    }
    pop_admitted(s, s->pend_query, r);
    r->dev_bytes = need;
    s->queries.push_back(r);
  }
}

// Seeds of the requests of B whose batch positions overlap [lo, hi): calls
// fn(request, first seed of the request in range, seeds in range).
template <class F>
void for_range(const Batch& B, uint64_t lo, uint64_t hi, F fn) {
  size_t a = 0, b = B.reqs.size();
  while (b - a > 1) {  // the last request starting at or before lo
    const size_t m = (a + b) / 2;
    if (B.reqs[m]->batch_off <= lo) a = m; else b = m;
  }
  for (size_t i = a; i < B.reqs.size() && B.reqs[i]->batch_off < hi; i++) {
    Req* r = B.reqs[i];
    const uint64_t r0 = std::max<uint64_t>(lo, r->batch_off), r1 = std::min<uint64_t>(hi, r->batch_off + r->q.nseeds);
    if (r1 > r0) fn(r, r0 - r->batch_off, r1 - r0);
  }
}

// Copies the batch's seeds into hs (pinned), sorts their ids by limb class
// into hi and sets cstart; in parts on the copy pool for large batches.
void gather_batch(collatz_server* s, Batch& B, uint32_t* hs, uint32_t* hi, uint32_t* cstart) {
  const uint64_t n = B.n;
  B.cls.resize(n);
  const int parts = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + COPY_PART_SEEDS - 1) / COPY_PART_SEEDS, 64));
  std::vector<uint32_t> cnt((size_t)parts * 5, 0);
  auto lo_of = [&](int p) { return n * (uint64_t)p / (uint64_t)parts; };
  s->copy_pool.run(parts, [&](int p) {
    const uint64_t lo = lo_of(p), hi_ = lo_of(p + 1);
    for_range(B, lo, hi_, [&](Req* r, uint64_t first, uint64_t m) {
      std::memcpy(hs + 8ull * (r->batch_off + first), r->q.seeds + 8ull * first, 32ull * m);
    });
    uint32_t* c = &cnt[(size_t)p * 5];
    for (uint64_t i = lo; i < hi_; i++) c[B.cls[i] = (uint8_t)traj_class(hs + 8 * i)]++;
  });
  // class-major positions: class j, then part p within it
  std::vector<uint32_t> fill((size_t)parts * 5);
  uint32_t off = 0;
  for (int j = 0; j < 5; j++) {
    cstart[j] = off;
    for (int p = 0; p < parts; p++) {
      fill[(size_t)p * 5 + j] = off;
      off += cnt[(size_t)p * 5 + j];
    }
  }
  cstart[5] = off;
  s->copy_pool.run(parts, [&](int p) {
    uint32_t* f = &fill[(size_t)p * 5];
    for (uint64_t i = lo_of(p); i < lo_of(p + 1); i++) hi[f[B.cls[i]]++] = (uint32_t)i;
  });
}

// Builds and enqueues one trajectory batch.  Returns 1 if one was launched,
// 0 if there are no queries waiting, negative on error.
int launch_batch(collatz_server* s, int bi) {
  if (s->queries.empty()) return 0;
  Batch& B = s->batches[bi];
  B.reqs.clear();
  uint64_t n = 0;
  while (!s->queries.empty() &&
         (B.reqs.empty() || n + s->queries.front()->q.nseeds <= s->cfg.traj_batch_seeds)) {
    Req* r = s->queries.front();
    s->queries.pop_front();
    r->batch_off = (uint32_t)n;
    n += r->q.nseeds;
    B.reqs.push_back(r);
  }
  collatz_ctx* c = s->ctx;
  B.n = (uint32_t)n;
  // host: seeds into pinned memory, class lists (region j holds class j's
  // own seeds followed by room for every seed of the narrower classes)
  const BatchLayout L(n);
  cudaError_t e = B.h_in.ensure(L.in_bytes);
  if (!e) e = B.h_out.ensure(L.out_bytes);
  if (e) return set_cuda_error(c, e, "server batch buffers");
  char* h = B.h_in.as<char>();
  TrajAllArgs a;
  gather_batch(s, B, reinterpret_cast<uint32_t*>(h), reinterpret_cast<uint32_t*>(h + L.o_idx), a.cstart);
  std::memset(h + L.o_cnt, 0, 64);
  // device: one block from the server's pool, freed in stream order
  const uint64_t bytes = L.o_out + L.out_bytes;
  cudaStream_t st = s->sb;
  void* block = nullptr;
  e = cudaMallocFromPoolAsync(&block, bytes, s->pool, st);
  if (e) return set_cuda_error(c, e, "server batch allocation");
  {
    uint64_t promised = 0;
    for (Req* r : B.reqs) promised += r->dev_bytes;
    std::lock_guard<std::mutex> g(s->mb);
    s->promised -= std::min(s->promised, promised);
    s->launched += promised;
  }
  char* d = static_cast<char*>(block);
  e = cudaMemcpyAsync(d, h, L.in_bytes, cudaMemcpyHostToDevice, st);
  if (!e) {
    // every limb class in one launch: a seed that needs more limbs is re-run by its thread
    a.seeds = reinterpret_cast<const uint32_t*>(d);
    a.index = reinterpret_cast<const uint32_t*>(d + L.o_idx);
    a.st = reinterpret_cast<unsigned long long*>(d + L.o_out + L.r_st);
    a.exc = reinterpret_cast<uint32_t*>(d + L.o_out + L.r_exc);
    a.status = reinterpret_cast<uint32_t*>(d + L.o_out + L.r_status);
    a.cursor = reinterpret_cast<uint32_t*>(d + L.o_cnt);
    a.iter_cap = c->iter_cap;
    const uint32_t grid = (uint32_t)std::min<uint64_t>((n + 127) / 128, (uint64_t)c->sm_count * 8);
    e = launch_traj_all(a, grid, st);
  }
  if (!e) e = cudaMemcpyAsync(B.h_out.p, d + L.o_out, L.out_bytes, cudaMemcpyDeviceToHost, st);
  const cudaError_t ef = cudaFreeAsync(block, st);
  if (!e) e = ef;
  if (!e) e = cudaEventRecord(B.done, st);
  if (e) return set_cuda_error(c, e, "server batch launch");
  B.busy = true;
  s->batch_order.push_back(bi);
  std::lock_guard<std::mutex> g(s->mu);
  s->info.traj_batches++;
  return 1;
}

void complete_batch(collatz_server* s, int bi) {
  Batch& B = s->batches[bi];
  // results into the callers' buffers, in parts on the copy pool for large batches
  const uint64_t n = B.n;
  const BatchLayout L(n);
  const char* h = B.h_out.as<char>();
  const uint64_t* h_st = reinterpret_cast<const uint64_t*>(h + L.r_st);
  const uint32_t* h_exc = reinterpret_cast<const uint32_t*>(h + L.r_exc);
  const uint32_t* h_status = reinterpret_cast<const uint32_t*>(h + L.r_status);
  const int parts = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + COPY_PART_SEEDS - 1) / COPY_PART_SEEDS, 64));
  s->copy_pool.run(parts, [&](int p) {
    for_range(B, n * (uint64_t)p / (uint64_t)parts, n * (uint64_t)(p + 1) / (uint64_t)parts,
              [&](Req* r, uint64_t first, uint64_t m) {
                const uint64_t o = r->batch_off + first;
                std::memcpy(r->q.stopping_time + first, h_st + o, 8 * m);
                std::memcpy(r->q.excursion + 16 * first, h_exc + 16 * o, 64 * m);
                std::memcpy(r->q.status + first, h_status + o, 4 * m);
              });
  });
  for (Req* r : B.reqs) {
    s->active[1]--;
    publish(s, r, COLLATZ_OK);
  }
  B.reqs.clear();
  B.busy = false;
  std::lock_guard<std::mutex> g(s->mu);
  s->info.traj_seeds += B.n;
}

// ---------------------------------------------------------------------
// worker loops
// ---------------------------------------------------------------------

// Fails every request a worker holds or that is queued for it (after a
// device error); the server then accepts no more requests.
void fail_worker(collatz_server* s, bool range_side, int rc) {
  std::vector<Req*> all;
  if (range_side) {
    all.assign(s->ranges.begin(), s->ranges.end());
    s->ranges.clear();
  } else {
    all.assign(s->queries.begin(), s->queries.end());
    s->queries.clear();
    for (Batch& B : s->batches) {
      all.insert(all.end(), B.reqs.begin(), B.reqs.end());
      B.reqs.clear();
    }
  }
  std::deque<Req*> pend;
  {
    std::lock_guard<std::mutex> g(s->mu);
    pend.swap(range_side ? s->pend_range : s->pend_query);
    s->stopping = true;
  }
  for (Req* r : all) {
    s->active[range_side ? 0 : 1]--;
    publish(s, r, rc);
  }
  for (Req* r : pend) publish(s, r, rc);
  s->cv_range.notify_all();
  s->cv_query.notify_all();
}

template <class Work>
void worker(collatz_server* s, bool range_side, Work work) {
  cudaSetDevice(s->ctx->device);
  double t[T_N] = {};
  std::deque<Req*>& pend = range_side ? s->pend_range : s->pend_query;
  std::condition_variable& cv = range_side ? s->cv_range : s->cv_query;
  for (;;) {
    Clock::time_point t_start = Clock::now();
    bool busy_device = false;
    {
      std::unique_lock<std::mutex> g(s->mu);
      if (s->stopping) {  // queued requests are not started after stop
        for (Req* r : pend) {
          r->status = COLLATZ_E_STATE;
          r->done_s = since(s->t0);
          s->done[r->ticket] = r;
          s->info.completed++;
        }
        pend.clear();
        s->cv_done.notify_all();
      }
      const bool held = range_side ? (!s->ranges.empty() || !s->slice_order.empty())
                                   : (!s->queries.empty() || !s->batch_order.empty());
      if (!held && s->stopping) return;
      if (!held && pend.empty()) cv.wait_for(g, std::chrono::milliseconds(50));
      s->info.loops++;
      for (int i = 0; i < T_N; i++) s->host_t[range_side ? 0 : 1][i] = t[i];
    }
    Clock::time_point tp = Clock::now();
    t[T_IDLE] += std::chrono::duration<double>(tp - t_start).count();
    const int rc = work(t, tp, busy_device);
    if (rc < 0) {
      cudaStreamSynchronize(range_side ? s->sa : s->sb);
      if (range_side) s->slice_order.clear(); else s->batch_order.clear();
      fail_worker(s, range_side, rc);
      return;
    }
    if (!rc) {  // nothing happened: wait for the device, a new request or a budget read
      const Clock::time_point tw = Clock::now();
      std::unique_lock<std::mutex> g(s->mu);
      cv.wait_for(g, std::chrono::microseconds(50));
      t[T_IDLE] += std::chrono::duration<double>(Clock::now() - tw).count();
    }
  }
}

void lap(double* t, int bucket, Clock::time_point& tp) {
  const Clock::time_point n = Clock::now();
  t[bucket] += std::chrono::duration<double>(n - tp).count();
  tp = n;
}

// One pass of a worker: admit, launch, complete.  Returns < 0 on a device
// error, 1 if anything happened, 0 otherwise (busy_device: work in flight).
int range_pass(collatz_server* s, double* t, Clock::time_point tp, bool& busy_device) {
  int did = 0;
  admit_ranges(s);
  lap(t, T_ADMIT, tp);
  for (int i = 0; i < SLICE_DEPTH; i++)
    if (!s->slices[i].busy) {
      const int rc = launch_slice(s, i);
      if (rc < 0) return rc;
      if (rc == 0) break;
      did = 1;
    }
  lap(t, T_BUILD, tp);
  while (!s->slice_order.empty()) {
    const cudaError_t q = cudaEventQuery(s->slices[s->slice_order.front()].done);
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) return set_cuda_error(s->ctx, q, "range slice");
    complete_slice(s, s->slice_order.front());
    s->slice_order.pop_front();
    did = 1;
  }
  lap(t, T_COMPLETE, tp);
  busy_device = !s->slice_order.empty();
  return did;
}

int query_pass(collatz_server* s, double* t, Clock::time_point tp, bool& busy_device) {
  int did = 0;
  admit_queries(s);
  lap(t, T_ADMIT, tp);
  for (int i = 0; i < BATCH_DEPTH; i++)
    if (!s->batches[i].busy) {
      const int rc = launch_batch(s, i);
      if (rc < 0) return rc;
      if (rc == 0) break;
      did = 1;
    }
  lap(t, T_BUILD, tp);
  while (!s->batch_order.empty()) {
    const cudaError_t q = cudaEventQuery(s->batches[s->batch_order.front()].done);
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) return set_cuda_error(s->ctx, q, "trajectory batch");
    complete_batch(s, s->batch_order.front());
    s->batch_order.pop_front();
    did = 1;
  }
  lap(t, T_COMPLETE, tp);
  busy_device = !s->batch_order.empty();
  return did;
}

void destroy(collatz_server* s) {
  if (!s) return;
  s->copy_pool.shutdown();
  if (s->ctx) {
    cudaSetDevice(s->ctx->device);
    if (s->sa) cudaStreamSynchronize(s->sa);
    if (s->sb) cudaStreamSynchronize(s->sb);
    for (Slice& S : s->slices) {
      S.d_segs.release();
      S.d_cursor.release();
      S.d_widen[0].release();
      S.d_widen[1].release();
      S.d_wcount.release();
      S.h_segs.release();
      S.h_recs.release();
      if (S.t0) cudaEventDestroy(S.t0);
      if (S.done) cudaEventDestroy(S.done);
    }
    for (Batch& B : s->batches) {
      B.h_in.release();
      B.h_out.release();
      if (B.done) cudaEventDestroy(B.done);
    }
    s->d_recs.release();
    if (s->sa) cudaStreamDestroy(s->sa);
    if (s->sb) cudaStreamDestroy(s->sb);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    collatz_destroy(s->ctx);
  }
  for (auto& kv : s->known) delete kv.second;
  delete s;
}

}  // namespace

extern "C" void collatz_server_config_default(collatz_server_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof *c);
  c->max_active = 256;
  c->slice_items = 1u << 19;  // ~1 ms of device work at k = 24
  c->hbm_reserve = 1ull << 30;
  c->traj_batch_seeds = 1u << 20;
}

extern "C" int collatz_server_start(const collatz_config* cfg, const collatz_server_config* scfg,
                                    collatz_server** out) {
  if (!out) return COLLATZ_E_ARG;
  *out = nullptr;
  collatz_server* s = new collatz_server();
  if (scfg) s->cfg = *scfg; else collatz_server_config_default(&s->cfg);
  if (s->cfg.max_active == 0 || s->cfg.max_active > MAX_ACTIVE_LIMIT || s->cfg.slice_items == 0 ||
      s->cfg.traj_batch_seeds == 0 || s->cfg.traj_batch_seeds > MAX_BATCH_SEEDS) {
    delete s;
    return COLLATZ_E_ARG;
  }
  int rc = collatz_create(cfg, &s->ctx);
  if (rc) {
    delete s;
    return rc;
  }
  collatz_ctx* c = s->ctx;
  auto fail = [&](cudaError_t e, const char* where) {
    set_cuda_error(c, e, where);
    destroy(s);
    return COLLATZ_E_CUDA;
  };
  DeviceScope dev_scope(c->device);
  cudaError_t e = dev_scope.err;
  if (e) return fail(e, "cudaSetDevice");
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  if ((e = cudaStreamCreateWithPriority(&s->sa, cudaStreamNonBlocking, lo))) return fail(e, "stream");
  if ((e = cudaStreamCreateWithPriority(&s->sb, cudaStreamNonBlocking, hi))) return fail(e, "stream");
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = c->device;
  if ((e = cudaMemPoolCreate(&s->pool, &props))) return fail(e, "cudaMemPoolCreate");
  uint64_t keep = 1ull << 30;  // idle pool memory kept for the next batches
  cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  if ((e = s->d_recs.ensure(sizeof(ReqRec) * s->cfg.max_active))) return fail(e, "server records");
  for (Slice& S : s->slices) {
    if ((e = S.d_cursor.ensure(sizeof(unsigned long long)))) return fail(e, "slice");
    if ((e = S.d_widen[0].ensure(sizeof(WidenEntry) * WIDEN_CAP))) return fail(e, "slice");
    if ((e = S.d_widen[1].ensure(sizeof(WidenEntry) * WIDEN_CAP))) return fail(e, "slice");
    if ((e = S.d_wcount.ensure(2 * sizeof(uint32_t)))) return fail(e, "slice");
    if ((e = cudaEventCreate(&S.t0))) return fail(e, "event");
    if ((e = cudaEventCreate(&S.done))) return fail(e, "event");
  }
  // Host and device staging is allocated here, once: growing a pinned or
  // device buffer later (cudaFreeHost / cudaFree synchronise the device,
  // large cudaMallocHost calls take milliseconds) would stall both workers.
  // per request: its segments and one threshold-scout index
  const size_t seg_bytes = (sizeof(RangeSeg) * SEGS_PER_REQ + sizeof(uint32_t)) * s->cfg.max_active;
  for (Slice& S : s->slices) {
    if ((e = S.d_segs.ensure(seg_bytes))) return fail(e, "slice");
    if ((e = S.h_segs.ensure(seg_bytes))) return fail(e, "slice");
    if ((e = S.h_recs.ensure(sizeof(ReqRec) * s->cfg.max_active))) return fail(e, "slice");
  }
  const uint64_t nb = s->cfg.traj_batch_seeds;
  for (Batch& B : s->batches) {
    if ((e = cudaEventCreateWithFlags(&B.done, cudaEventDisableTiming))) return fail(e, "event");
    if ((e = B.h_in.ensure(BatchLayout(nb).in_bytes))) return fail(e, "batch");
    if ((e = B.h_out.ensure(BatchLayout(nb).out_bytes))) return fail(e, "batch");
    B.cls.reserve(nb);
  }
  // the query pool grown to two full batches now (growing it under load took milliseconds)
  {
    const BatchLayout L(nb);
    void* blk[BATCH_DEPTH] = {};
    for (void*& b : blk)
      if (!e) e = cudaMallocFromPoolAsync(&b, L.o_out + L.out_bytes, s->pool, s->sb);
    for (void* b : blk)
      if (b) cudaFreeAsync(b, s->sb);
    const cudaError_t es = cudaStreamSynchronize(s->sb);
    if (!e) e = es;
    if (e) return fail(e, "query pool");
  }
  size_t fr = 0;
  if ((e = cudaMemGetInfo(&fr, &s->total_mem))) return fail(e, "cudaMemGetInfo");
  refresh_budget(s);
  for (uint32_t i = s->cfg.max_active; i-- > 0;) s->free_slots.push_back(i);
  // helpers for the query path's host copies: up to 7, half the host's threads at most
  s->copy_pool.start((int)std::min(7u, std::max(1u, std::thread::hardware_concurrency() / 2) - 1u));
  s->t0 = Clock::now();
  s->thr_range = std::thread([s] { worker(s, true, [s](double* t, Clock::time_point tp, bool& b) {
                                       return range_pass(s, t, tp, b);
                                     }); });
  s->thr_query = std::thread([s] { worker(s, false, [s](double* t, Clock::time_point tp, bool& b) {
                                       return query_pass(s, t, tp, b);
                                     }); });
  s->thr_budget = std::thread([s] { budget_loop(s); });
  *out = s;
  return COLLATZ_OK;
}

extern "C" int collatz_server_submit(collatz_server* s, const collatz_request* q, uint64_t* ticket) {
  if (!s || !q || !ticket) return COLLATZ_E_ARG;
  if (q->kind == COLLATZ_REQ_RANGE) {
    const uint32_t k = q->range.k;
    if (k && (k < 8 || k > 34)) return COLLATZ_E_ARG;
    const unsigned __int128 o = ((unsigned __int128)q->range.offset[1] << 64) | q->range.offset[0];
    if (q->range.size > (1ull << 48) || o + q->range.size > ((unsigned __int128)1 << 96)) return COLLATZ_E_LIMIT;
  } else if (q->kind == COLLATZ_REQ_TRAJECTORY) {
    if (!q->nseeds || !q->seeds || !q->stopping_time || !q->excursion || !q->status) return COLLATZ_E_ARG;
    if (q->nseeds > s->cfg.traj_batch_seeds) return COLLATZ_E_LIMIT;
  } else {
    return COLLATZ_E_ARG;
  }
  Req* r = new Req();
  r->q = *q;
  r->submit_s = since(s->t0);
  const bool is_range = q->kind == COLLATZ_REQ_RANGE;
  {
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stopping) {
      delete r;
      return COLLATZ_E_STATE;
    }
    r->ticket = s->next_ticket++;
    s->known[r->ticket] = r;
    (is_range ? s->pend_range : s->pend_query).push_back(r);
    s->info.submitted++;
  }
  (is_range ? s->cv_range : s->cv_query).notify_one();
  *ticket = r->ticket;
  return COLLATZ_OK;
}

extern "C" int collatz_server_wait(collatz_server* s, uint64_t ticket, double timeout_s, collatz_response* resp) {
  if (!s) return COLLATZ_E_ARG;
  std::unique_lock<std::mutex> g(s->mu);
  if (!s->known.count(ticket)) return COLLATZ_E_ARG;
  auto ready = [&] { return s->done.count(ticket) != 0; };
  if (timeout_s < 0) {
    s->cv_done.wait(g, ready);
  } else if (!s->cv_done.wait_for(g, std::chrono::duration<double>(timeout_s), ready)) {
    return COLLATZ_E_TIMEOUT;
  }
  Req* r = s->done[ticket];
  s->done.erase(ticket);
  s->known.erase(ticket);
  g.unlock();
  if (resp) {
    std::memset(resp, 0, sizeof *resp);
    resp->ticket = r->ticket;
    resp->status = r->status;
    resp->kind = r->q.kind;
    resp->range = r->res;
    resp->range.status = r->status;
    resp->submit_s = r->submit_s;
    resp->admit_s = r->admit_s;
    resp->done_s = r->done_s;
  }
  const int st = r->status;
  delete r;
  return st;
}

extern "C" int collatz_server_info(collatz_server* s, collatz_server_info_t* info) {
  if (!s || !info) return COLLATZ_E_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  *info = s->info;
  info->pending = (uint32_t)(s->pend_range.size() + s->pend_query.size());
  info->active = s->active[0].load() + s->active[1].load();
  info->host_admit_s = s->host_t[0][T_ADMIT] + s->host_t[1][T_ADMIT];
  info->host_slice_s = s->host_t[0][T_BUILD];
  info->host_batch_s = s->host_t[1][T_BUILD];
  info->host_complete_s = s->host_t[0][T_COMPLETE] + s->host_t[1][T_COMPLETE];
  info->host_idle_s = s->host_t[0][T_IDLE] + s->host_t[1][T_IDLE];
  return COLLATZ_OK;
}

extern "C" int collatz_server_stop(collatz_server* s) {
  if (!s) return COLLATZ_E_ARG;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stopping = true;
  }
  s->cv_range.notify_all();
  s->cv_query.notify_all();
  if (s->thr_range.joinable()) s->thr_range.join();
  if (s->thr_query.joinable()) s->thr_query.join();
  {
    std::lock_guard<std::mutex> g(s->mb);
    s->budget_stop = true;
  }
  s->cv_budget.notify_all();
  if (s->thr_budget.joinable()) s->thr_budget.join();
  destroy(s);
  return COLLATZ_OK;
}
