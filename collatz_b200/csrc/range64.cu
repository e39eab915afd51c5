// range64.cu -- range verification with 64-bit values: the kernel for
// launches whose seeds all lie below 2^52 (a context's limb-width cutoff,
// chosen by the autotuner).  It verifies the same seeds with the same
// results as k_range (range.cu) -- same work items, survivor table, mod-9
// sieve, k-step jump, threshold prefilters, offers and widening -- but a
// seed's state is one 64-bit value instead of four 32-bit limbs:
//
//   * a queue entry is 16 bytes: v = T^s(n) + 1 and n, with the item slot,
//     the excursion-candidate flag and s packed into the bits above n;
//   * a run pair on a value below 2^59 is one 64-bit odd run (capped at 7
//     steps, so the value stays below 2^64) and one 64-bit even run;
//   * a lane whose value reaches 2^59 runs its run pairs on four limbs
//     (128 bits) until it comes back below -- lane by lane, so the other
//     lanes keep the 64-bit pair -- and a value that could leave 2^128 sends
//     the seed to the widen list (re-run from scratch with 6 and 8 limbs);
//   * at expansion every seed takes up to M run pairs in its lane; the seeds
//     still running are then packed into lanes and take up to M2 more, so
//     that the warp does not step every entry's pairs for the few that need
//     them; the rest go to the queue;
//   * the run loop takes one warp vote per step for all of its rare events (a
//     value at or above 2^59, an excursion candidate, a finish that may
//     offer) when V is set;
//   * idle lanes take queued seeds at the first step of each pass of R steps,
//     and at the later steps only when at least PT lanes are idle: a pop costs
//     the warp the same instructions for one idle lane as for 32;
//   * with J > 0, a lane whose value is far from its seed and from the
//     excursion threshold takes J steps at once from a 2^J-entry table in
//     shared memory (rs:111-123 and rs:321-341 give the jump-table form,
//     v -> (v >> J) 3^f(r) + T^J(r); here bit lengths prove that no step of
//     the J can descend or reach the threshold, so results stay exact).
#include <cuda_runtime.h>

#include "range_shared.cuh"

namespace cz {

constexpr u32 R64_WARPS = 8;              // warps per block
constexpr u32 Q64 = 128;                  // queue entries per warp (power of two, >= 32 R + one item)
constexpr u64 FAST_LIMIT = 1ull << 59;    // a 64-bit run pair needs the value below this
constexpr u32 SEED_BITS_64 = 48;          // seeds must lie below 2^48 (n fits 16 bits of the entry's word 3)
constexpr u32 ST_ENTRY_MAX = 1023;        // steps stored in a queue entry (10 bits)

// Per-warp state in shared memory.  Queue entry: x, y = v = T^s(n) + 1 (low,
// high word); z = n bits 0..31; w = n bits 32..47 | item slot << 16 |
// candidate << 21 | s << 22 (s <= 1023).
struct Warp64 {
  uint4 q[Q64];
  uint4 ring[RR];           // per item slot: request, sigma threshold, excursion gate (lo, hi) as a value
  u32 ring_end[RR];         // per item slot: queue position after the item's last seed
  uint4 stage[RANGE_ITEM];  // survivor entries of the staged item (cp.async)
  u32 e[4][32];             // per lane: seed-local max excursion
  u32 pe[4][32];            // per lane: excursion of a pending offer
  u32 c[5][32];             // per lane: pending offer [0] sigma [1..3] seed [4] request
  RangeSeg seg;             // cached segment
  StagedItem nxt;
  ull item, claim_hi, seg_lo, seg_hi, qi, acc_seeds, acc_items;
  u32 chunk, since_thr, ring_seq, thr_bl, pad0, pad1;
};

// The excursion gate of a threshold window (bits 32..95 of the threshold,
// all ones when it is >= 2^96) as a 64-bit value: a value v (in +1 space)
// is a candidate when v >= gate64.  Thresholds of 2^64 and more give all
// ones, which no 64-bit run-pair value reaches.
__device__ __forceinline__ u64 gate64_of(u64 window) { return (window >> 32) ? ~0ull : (window << 32); }

__device__ __forceinline__ u32 bitlen64(u64 x) { return x ? 64u - __clzll(x) : 0u; }

// Drops pending offers that another pending lane of the same request beats
// (larger, or equal with a smaller seed), so that one offer per request and
// kind remains; all lanes call it together.
__device__ __noinline__ u32 drop_dominated64(Warp64& W, u32 lane, u32 pend, u32 pm) {
  const u32 m1 = __ballot_sync(FULL, pend & 1u), m2 = __ballot_sync(FULL, pend & 2u);
  __syncwarp();
  if (pend) {
    const u32 rq = W.c[4][lane], s0 = W.c[1][lane], s1 = W.c[2][lane];
    for (u32 m = pm & ~(1u << lane); m; m &= m - 1) {
      const u32 j = __ffs(m) - 1;
      if (W.c[4][j] != rq) continue;
      const u32 t0 = W.c[1][j], t1 = W.c[2][j];
      const bool j_smaller = (t1 != s1) ? (t1 < s1) : (t0 < s0);
      if ((pend & 1u) && ((m1 >> j) & 1u)) {
        const u32 sj = W.c[0][j], si = W.c[0][lane];
        if (sj > si || (sj == si && j_smaller)) pend &= ~1u;
      }
      if ((pend & 2u) && ((m2 >> j) & 1u)) {
        int c = 0;
#pragma unroll
        for (int i = 3; i >= 0; i--)
          if (c == 0) c = (W.pe[i][j] > W.pe[i][lane]) ? 1 : ((W.pe[i][j] < W.pe[i][lane]) ? -1 : 0);
        if (c > 0 || (c == 0 && j_smaller)) pend &= ~2u;
      }
    }
  }
  __syncwarp();
  return pend;
}

struct Stats64 {
  u32 pairs = 0, fast = 0, slow_e = 0, replay = 0, jump = 0, pop = 0, exp = 0, pass = 0, offer = 0, win = 0,
      tab = 0, xpairs = 0, xfin = 0;
};

// Up to C jumps of JW steps each from the table s_win, while bit lengths prove
// that none of the JW steps can descend below the seed (bitlen(n) = nbl) or
// reach the excursion threshold (whose bit length is at least thr_bl; every
// value stays below 2^(thr_bl - 1)).  v = T^s(n) + 1 and st = s are updated.
template <int JW, int C, bool STATS>
__device__ __forceinline__ void chain_windows(u64& v, u32& st, u32 nbl, u32 thr_bl, const u32* s_win,
                                              const u32* s_pow3, Stats64& X) {
#pragma unroll
  for (int c = 0; c < C; c++) {
    const u64 x = v - 1;
    const u32 te = s_win[(u32)x & ((1u << JW) - 1u)];
    const u64 a = x >> JW;
    const u32 abl = bitlen64(a), glen = (te >> 22) & 31u, hlen = te >> 27;
    if (!((abl != 0) & (abl + glen >= nbl + 2u) & (abl + hlen < thr_bl) & (abl + hlen <= 62u))) break;
    v = a * s_pow3[(te >> 18) & 15u] + (te & 0x3FFFFu) + 1u;
    st += (u32)JW;
    if (STATS) X.win++;
  }
}

// Up to M run pairs of a seed taken at expansion, with every lane busy.  A
// pair is kept only in the common case: the value stays below 2^59, no value
// reaches the excursion gate G, and the seed either does not descend or
// descends with a stopping time below the threshold thr_st (it can then
// change no maximum).  Otherwise the pair is left undone for the run loop,
// which handles every case.  Returns false when the seed finished here.
template <int M, bool STATS>
__device__ __forceinline__ bool first_pairs(u64& v, u32& st, u64 n, u64 G, u32 thr_st, const u32* s_pow3,
                                            Stats64& X) {
#pragma unroll
  for (int m = 0; m < M; m++) {
    if (v >= FAST_LIMIT) break;
    const u32 a = ctz32((u32)v | 0x80u);
    const u64 x = (v >> a) * s_pow3[a] - 1;
    if (x + 1 >= G) break;  // an excursion candidate: the loop takes this pair
    const u32 b = ctz32((u32)x | 0x80000000u);
    const u64 w = x >> b;
    const u32 st2 = st + a + b;
    if (w < n) {  // descends in this pair (b = 0 leaves x, which is above n)
      if (st2 >= thr_st) break;  // sigma may reach the maximum: the loop takes this pair
      if (STATS) X.xfin++;
      return false;
    }
    v = w + 1;
    st = st2;
    if (STATS) X.xpairs++;
  }
  return true;
}

// Second stage of the run pairs taken at expansion: the seeds that the first
// stage kept sit in W.q[tail, tail + total); each takes up to M2 more pairs
// (the same rules as first_pairs, so the two stages give exactly what
// first_pairs<M + M2> gives) and those still running are written back,
// compacted, from tail.  Packing the survivors into lanes first keeps the
// warp from stepping every entry's M + M2 pairs for the few that need them.
// Returns the number kept.  Warp-uniform.
template <int M2, bool STATS>
__device__ __forceinline__ u32 second_pairs(Warp64& W, u32 lane, u32 tail, u32 total, u32 slot, u64 G, u32 thr_st,
                                            const u32* s_pow3, Stats64& X) {
  u32 kept = 0;
  for (u32 base = 0; base < total; base += 32) {
    const bool has = base + lane < total;
    const uint4 e = has ? W.q[(tail + base + lane) & (Q64 - 1)] : make_uint4(0u, 0u, 0u, 0u);
    __syncwarp();  // every entry of this round is read before any is overwritten
    u64 v = ((u64)e.y << 32) | e.x;
    const u64 n = ((u64)(e.w & 0xFFFFu) << 32) | e.z;
    u32 st = e.w >> 22;
    const bool keep = has && first_pairs<M2, STATS>(v, st, n, G, thr_st, s_pow3, X);
    const u32 bk = __ballot_sync(FULL, keep);
    if (keep) {  // kept <= base: the slot written was read in this round or an earlier one
      const u32 cand = v >= G ? 1u : 0u;
      W.q[(tail + kept + __popc(bk & lanemask_lt())) & (Q64 - 1)] =
          make_uint4((u32)v, (u32)(v >> 32), (u32)n, (u32)(n >> 32) | (slot << 16) | (cand << 21) | (st << 22));
    }
    kept += __popc(bk);
    __syncwarp();
  }
  return kept;
}

// Expands the staged item into the warp's queue from position tail (see
// expand_one in range.cu for the rules; this is its 64-bit form).  Seeds are
// below 2^52, so the block q is below 2^(52-k) and n = q 2^k + r is one
// 64-bit word; the jump q 3^f + c is taken when it fits 63 bits, else the
// seed replays its first k steps from v = n + 1.  Warp-uniform.
template <int JW, int C, int M, int M2, bool NQ, bool STATS>
__device__ __forceinline__ bool expand64(Warp64& W, const RangeArgs& A, const uint4* __restrict__ T, u32 lane, u32 k,
                                         u32 k9, const unsigned long long* s_p3, const u32* s_pow3, const u32* s_win,
                                         u32 head, u32& tail, bool& exhausted, u32& w_thr_st, u32& w_req, u64& w_gate,
                                         Stats64& X) {
  if ((int)(W.ring_end[W.ring_seq & (RR - 1)] - head) > 0) return false;
  cp_async_wait_all();  // this lane's copies of the staged item
  __syncwarp();
  const StagedItem it = W.nxt;
  if (!it.valid) {
    exhausted = true;
    return true;
  }
  uint4 e[RANGE_ITEM / 32];
  if (it.kind == 0) {
#pragma unroll
    for (u32 j = 0; j < RANGE_ITEM / 32; j++) e[j] = W.stage[j * 32 + lane];
  }
  __syncwarp();
  stage_next(W, W.stage, A, T, lane);  // the following item's copies overlap with this expansion
  const u32 rq = it.req;
  if (rq != w_req || ++W.since_thr >= 64) {  // thresholds of the request, refreshed now and then
    ull sk = 0, ek = 0;
    if (lane == 0 && rq != w_req && w_req != 0xFFFFFFFFu) {
      if (W.acc_seeds) atomicAdd(&A.recs[w_req].seeds, W.acc_seeds);
      atomicAdd(&A.recs[w_req].items_done, W.acc_items);
    }
    if (lane == 0) {
      sk = *(volatile ull*)&A.recs[rq].st_key;
      ek = *(volatile ull*)&A.recs[rq].e_key;
    }
    sk = __shfl_sync(FULL, sk, 0);
    ek = __shfl_sync(FULL, ek, 0);
    u32 t[4];
    key_decode<4>(ek, t);
    if (rq != w_req) {
      w_thr_st = 0;
      w_gate = 0;
    }
    w_thr_st = max(w_thr_st, (u32)min(sk, 0xFFFFFFFFull));
    w_gate = max(w_gate, gate_window(t[1], t[2], t[3]));
    __syncwarp();
    if (lane == 0) {
      if (rq != w_req) W.acc_seeds = W.acc_items = W.thr_bl = 0;
      W.thr_bl = max(W.thr_bl, (u32)(ek >> 54));
      W.since_thr = 0;
    }
    w_req = rq;
    __syncwarp();
  }
  const u32 w_thr_bl = W.thr_bl;
  const u64 G = gate64_of(w_gate);
  const u32 slot = W.ring_seq & (RR - 1);
  u32 mask = 0, total, seeds;
  if (it.kind == 0) {
    const u64 q = it.q_lo;  // < 2^(52 - k)
    const u64 qk = q << k;
    const u32 nbl = bitlen64(q) + k;
    if (it.mod9) {  // segments of whole kept classes (the usual case) need no per-entry test
      const u32 b9 = (mod9_96((u32)q, (u32)(q >> 32), 0u) * k9) % 9u;
#pragma unroll
      for (u32 j = 0; j < RANGE_ITEM / 32; j++) {
        if (it.sbase + j * 32 + lane < it.send) {
          u32 x = b9 + ((e[j].y >> 16) & 0xFFu);
          x = (x >= 9u) ? x - 9u : x;
          if ((KEEP9 >> x) & 1u) mask |= 1u << j;
        }
      }
    } else {
#pragma unroll
      for (u32 j = 0; j < RANGE_ITEM / 32; j++)
        if (it.sbase + j * 32 + lane < it.send) mask |= 1u << j;
    }
    // each entry in turn: its seed's start state (the k-step jump, up to C windows of JW
    // steps, up to M run pairs), then one ballot places the lanes' seeds in the queue
    seeds = __reduce_add_sync(FULL, __popc(mask));
    total = 0;
#pragma unroll
    for (u32 j = 0; j < RANGE_ITEM / 32; j++) {
      const u32 f = (e[j].y >> 8) & 0xFFu, emax = e[j].y >> 24;
      const u64 n = qk | e[j].x | ((u64)(e[j].y & 0xFFu) << 32);
      u64 v = n + 1;
      u32 st = 0;
      // T^0..T^k(n) < 2^(bitlen(n) + 1 + emax): skip them when that is below the excursion
      // threshold, else replay the first k steps exactly
      if (((mask >> j) & 1u) && nbl + 1 + emax < w_thr_bl) {
        const u64 p = s_p3[f];
        u64 lo, hi;
        if (NQ && (q >> 32) == 0) {  // warp-uniform: q 2^32-narrow, two wide multiply-adds
          const u64 t = (u64)(u32)q * (u32)p;
          const u64 u = (u64)(u32)q * (u32)(p >> 32) + (t >> 32);
          lo = (u << 32) | (u32)t;
          hi = u >> 32;
        } else {
          lo = q * p;
          hi = __umul64hi(q, p);
        }
        const u64 vv = lo + (((u64)e[j].w << 32) | e[j].z);
        if ((hi == 0) & (vv >= lo) & (vv < (1ull << 63))) {
          v = vv;
          st = k;
          if (STATS) X.jump++;
          chain_windows<JW, C, STATS>(v, st, nbl, w_thr_bl, s_win, s_pow3, X);
        }
      }
      if (STATS && ((mask >> j) & 1u) && st == 0) X.replay++;
      const bool keep = ((mask >> j) & 1u) && first_pairs<M, STATS>(v, st, n, G, w_thr_st, s_pow3, X);
      const u32 bk = __ballot_sync(FULL, keep);
      if (keep) {
        const u32 cand = v >= G ? 1u : 0u;
        W.q[(tail + total + __popc(bk & lanemask_lt())) & (Q64 - 1)] =
            make_uint4((u32)v, (u32)(v >> 32), (u32)n, (u32)(n >> 32) | (slot << 16) | (cand << 21) | (st << 22));
      }
      total += __popc(bk);
    }
  } else {
    // integers below 2^k: [d, d + 64) of [q_lo, d_hi), no residue sieve
    const ull d = it.q_lo + 2ull * lane;
#pragma unroll
    for (u32 j = 0; j < 2; j++) {
      const ull n = d + j;
      if (n < it.d_hi && n >= 2 && (!it.mod9 || ((KEEP9 >> (u32)(n % 9u)) & 1u))) mask |= 1u << j;
    }
    seeds = __reduce_add_sync(FULL, __popc(mask));
    total = 0;
#pragma unroll
    for (u32 j = 0; j < 2; j++) {
      const ull n = d + j;
      u64 v = n + 1;
      u32 st = 0;
      const bool keep = ((mask >> j) & 1u) && first_pairs<M, STATS>(v, st, n, G, w_thr_st, s_pow3, X);
      const u32 bk = __ballot_sync(FULL, keep);
      if (keep) {
        const u32 cand = v >= G ? 1u : 0u;
        W.q[(tail + total + __popc(bk & lanemask_lt())) & (Q64 - 1)] =
            make_uint4((u32)v, (u32)(v >> 32), (u32)n, (u32)(n >> 32) | (slot << 16) | (cand << 21) | (st << 22));
      }
      total += __popc(bk);
    }
  }
  __syncwarp();
  if (M2 > 0) total = second_pairs<M2, STATS>(W, lane, tail, total, slot, G, w_thr_st, s_pow3, X);
  if (lane == 0) {
    W.ring[slot] = make_uint4(rq, w_thr_st, (u32)G, (u32)(G >> 32));
    W.ring_end[slot] = tail + total;
    W.ring_seq++;
    W.acc_seeds += seeds;
    W.acc_items++;
  }
  if (STATS) X.exp++;
  tail += total;
  __syncwarp();
  return true;
}

template <int R, int MINB, int J, int JW, int C, int M, int M2, bool V, int PT, bool NQ, bool STATS>
__global__ void __launch_bounds__(R64_WARPS * 32, MINB) k_range64(const RangeArgs A) {
  // a queued seed's steps: k <= 34, C windows of JW steps, M run pairs of at most 7 + 31 steps
  static_assert(34 + C * JW + (M + M2) * 38 <= ST_ENTRY_MAX, "the step count of a queue entry has 10 bits");
  static_assert(Q64 >= 32 * R + RANGE_ITEM, "a refill may leave 32 R - 1 seeds queued and add one item");
  extern __shared__ __align__(16) unsigned char range64_smem[];
  Warp64* S = reinterpret_cast<Warp64*>(range64_smem);
  __shared__ unsigned long long s_p3[41];
  __shared__ u32 s_pow3[16];
  __shared__ u32 s_win[1u << JW];
  __shared__ u32 s_jt[J ? (1u << J) : 1];
  build_step_table(s_win, (u32)JW);
  if (J) build_step_table(s_jt, (u32)J);
  const u32 lane = lane_id();
  Warp64& W = S[threadIdx.x >> 5];
  if (threadIdx.x < 41) {
    unsigned long long p = 1;
    for (u32 i = 0; i < threadIdx.x; i++) p *= 3;
    s_p3[threadIdx.x] = p;
    if (threadIdx.x < 16) s_pow3[threadIdx.x] = (u32)p;
  }
  if (lane == 0) {
    W.item = ~0ull;
    W.claim_hi = 0;
    W.seg_lo = 1;
    W.seg_hi = 0;
    W.qi = W.acc_seeds = W.acc_items = 0;
    W.chunk = W.since_thr = W.ring_seq = W.thr_bl = 0;
    W.nxt.valid = 0;
  }
  W.ring_end[lane] = 0;  // RR == 32: one slot per lane
  __syncthreads();

  const u32 k = A.k;
  const u32 k9 = (u32)((1ull << (k % 6)) % 9ull);  // 2^k mod 9 (2^6 = 1 mod 9)
  const uint4* __restrict__ T = reinterpret_cast<const uint4*>(A.table);
  stage_next(W, W.stage, A, T, lane);
  Stats64 X;
  ull t_offer = 0, t_refill = 0, t_lanes = 0, t_mark = 0;

  // ---- warp-uniform state ----
  u32 head = 0, tail = 0;  // queued seeds [head, tail)
  bool exhausted = false;
  u32 w_thr_st = 0, w_req = 0xFFFFFFFFu;
  u64 w_gate = 0;  // excursion threshold window, bits 32..95 (all ones when it is >= 2^96)
  // ---- lane state ----
  u64 v = 0, vh = 0, n = 0, G = 0;  // value (+1 space) bits 0..63 and 64..127, seed, excursion gate
  u32 st = 0, req = 0, thr_st = 0, pend = 0;
  bool active = false, evalid = false;

  if (STATS) t_mark = clock64();
  for (;;) {
    if (STATS) {
      X.pass++;
      const ull now = clock64();
      t_lanes += now - t_mark;
      t_mark = now;
    }
    // ---- warp-synchronous part: offers of finished seeds (rare), refill, exit ----
    u32 pm = __ballot_sync(FULL, pend != 0);
    if (pm) {
      if (pm & (pm - 1)) {
        pend = drop_dominated64(W, lane, pend, pm);
        pm = __ballot_sync(FULL, pend != 0);
      }
      while (pm) {
        const u32 leader = __ffs(pm) - 1;
        const u32 lp = __shfl_sync(FULL, pend, leader), lreq = W.c[4][leader];
        if (lane == leader) {
          const u32 seed[4] = {W.c[1][lane], W.c[2][lane], W.c[3][lane], 0};
          if (STATS) X.offer++;
          if (pend & 1u) rec_offer_st(A.recs + lreq, W.c[0][lane], seed);
          if (pend & 2u) {
            const u32 e4[4] = {W.pe[0][lane], W.pe[1][lane], W.pe[2][lane], W.pe[3][lane]};
            rec_offer_e<4>(A.recs + lreq, e4, seed);
          }
          pend = 0;
        }
        __syncwarp();
        if (lreq == w_req) {  // an offered value is a lower bound of the request's maximum
          if (lp & 1u) w_thr_st = max(w_thr_st, W.c[0][leader]);
          if (lp & 2u) {
            const u32 e1 = W.pe[1][leader], e2 = W.pe[2][leader], e3 = W.pe[3][leader];
            w_gate = max(w_gate, gate_window(e1, e2, e3));
            const u32 t = e3 ? e3 : (e2 ? e2 : e1);
            const u32 bl = t ? (e3 ? 96u : (e2 ? 64u : 32u)) + 32u - __clz(t) : 0u;
            if (lane == 0) W.thr_bl = max(W.thr_bl, bl > 0 ? bl - 1 : 0u);
          }
        }
        pm &= pm - 1;
      }
    }
    if (STATS) {
      const ull now = clock64();
      t_offer += now - t_mark;
      t_mark = now;
    }
    // ---- refill: keep 32 R seeds queued (each lane takes at most R per pass) ----
    while (tail - head < 32u * R && !exhausted) {
      if (!expand64<JW, C, M, M2, NQ, STATS>(W, A, T, lane, k, k9, s_p3, s_pow3, s_win, head, tail, exhausted, w_thr_st, w_req,
                           w_gate, X))
        break;
    }
    __syncwarp();
    if (STATS) {
      const ull now = clock64();
      t_refill += now - t_mark;
      t_mark = now;
    }
    if (exhausted && tail == head && __ballot_sync(FULL, active) == 0) break;

#pragma unroll
    for (int r = 0; r < R; r++) {
      // The common path of a step has no lane-dependent branch: idle lanes take queued
      // seeds and active lanes run a 64-bit run pair with predicated code; the rare
      // events -- a value at or above 2^59, an excursion candidate, a finish that may
      // have to offer -- run behind warp-uniform votes.
      {
        const bool idle = !active && !pend;
        const u32 want = __ballot_sync(FULL, idle);
        // the first step of a pass refills every idle lane; the later ones only when at
        // least PT lanes are idle (PT <= 1: whenever one is)
        if (want && (r == 0 || PT <= 1 || __popc(want) >= PT)) {
          const u32 avail = tail - head;
          const u32 rank = __popc(want & lanemask_lt());
          const bool take = idle && rank < avail;
          const uint4 e = W.q[(head + rank) & (Q64 - 1)];
          const uint4 g = W.ring[(e.w >> 16) & 31u];
          const bool mine = g.x == w_req;  // the warp's thresholds are the freshest
          v = take ? (((u64)e.y << 32) | e.x) : v;
          vh = take ? 0ull : vh;
          n = take ? ((((u64)(e.w & 0xFFFFu)) << 32) | e.z) : n;
          st = take ? (e.w >> 22) : st;
          req = take ? g.x : req;
          thr_st = take ? (mine ? w_thr_st : g.y) : thr_st;
          G = take ? (mine ? gate64_of(w_gate) : (((u64)g.w << 32) | g.z)) : G;
          const bool c0 = take && ((e.w >> 21) & 1u);
          evalid = take ? c0 : evalid;
          active = active || take;
          if (c0) {  // the start value T^s(n) = v - 1 is an excursion candidate (rare)
            const u64 x = v - 1;
            W.e[0][lane] = (u32)x;
            W.e[1][lane] = (u32)(x >> 32);
            W.e[2][lane] = 0;
            W.e[3][lane] = 0;
          }
          if (STATS && take) X.pop++;
          head += min((u32)__popc(want), avail);
        }
      }
      bool jstep = false;
      if (J) {
        // J steps at once when they can neither descend nor reach the excursion gate: with
        // x = a 2^J + r, a g(r) <= T^i(x) < (a + 1) h(r) for every i <= J
        const u64 x = v - 1;
        const u32 te = s_jt[(u32)x & ((1u << J) - 1u)];
        const u64 a = x >> J;
        const u32 abl = bitlen64(a), glen = (te >> 22) & 31u, hlen = te >> 27;
        const bool jt = active & (vh == 0) & (v < FAST_LIMIT) & (abl != 0) & (abl + glen >= bitlen64(n) + 2u) &
                        (abl + hlen + 2u <= bitlen64(G)) & (abl + hlen <= 59u) & (st <= ST_CAP);
        const u64 vj = a * s_pow3[(te >> 18) & 15u] + (te & 0x3FFFFu) + 1u;
        if (jt) {  // this lane takes no run pair in this step
          v = vj;
          st += (u32)J;
          if (STATS) X.tab++;
        }
        jstep = jt;
      }
      bool fin = false;
      u32 b = 0;
      const bool slow = active & !jstep & ((vh != 0) | (v >= FAST_LIMIT));
      // four-limb run pair for a value at or above 2^59
      auto slow_pair = [&]() {
        u32 v0 = (u32)v, v1 = (u32)(v >> 32), v2 = (u32)vh, v3 = (u32)(vh >> 32);
        const u32 a = ctz32(v0 | 0x80u);
        odd_run4(v0, v1, v2, v3, a, pow3_le7(a));
        st += a;
        if (STATS) X.pairs++;
        // excursion / overflow gate: a value of 2^64 or more is always a candidate
        if (((v2 | v3) != 0) | ((((u64)v1 << 32) | v0) >= G)) {
          if (v3 >= OVF3) {
            // the next odd run could leave 128 bits: re-run this seed with wider limbs
            widen_seed(A, req, (u32)n, (u32)(n >> 32), 0u);
            active = false;
            return;
          }
          if (STATS) X.slow_e++;
          u32 xv[4];
          value_of<false>(v0, v1, v2, v3, xv);
          bool tk = !evalid;
          if (evalid)
            tk = lt96c(W.e[0][lane], W.e[1][lane], W.e[2][lane], xv[0], xv[1], xv[2]) ? (W.e[3][lane] <= xv[3])
                                                                                        : (W.e[3][lane] < xv[3]);
          if (tk) {
            W.e[0][lane] = xv[0];
            W.e[1][lane] = xv[1];
            W.e[2][lane] = xv[2];
            W.e[3][lane] = xv[3];
            evalid = true;
          }
        }
        v0 -= 1;  // v0 == 0 gives b == 0 below, and the borrow cancels against the +1
        b = ctz32(v0 | 0x80000000u);
        const u32 w0 = __funnelshift_r(v0, v1, b), w1 = __funnelshift_r(v1, v2, b);
        const u32 w2 = __funnelshift_r(v2, v3, b), w3 = v3 >> b;
        st += b;
        fin = (((w3 | w2) == 0) & (b != 0) & ((((u64)w1 << 32) | w0) < n)) | (st > ST_CAP);
        if (fin) {
          v = ((u64)v1 << 32) | v0;  // the value before the even run
          vh = ((u64)v3 << 32) | v2;
        } else {
          u32 y0 = w0 + 1, y1 = w1, y2 = w2, y3 = w3;
          add_carry3(y1, y2, y3, (y0 == 0) & (b != 0));
          v = ((u64)y1 << 32) | y0;
          vh = ((u64)y3 << 32) | y2;
        }
      };
      // an excursion candidate x of a 64-bit pair: keep it when it is the seed's largest value
      auto take_candidate = [&](u64 x) {
        if (STATS) X.slow_e++;
        const u64 ex = ((u64)W.e[1][lane] << 32) | W.e[0][lane];
        if (!evalid || (W.e[2][lane] == 0 && W.e[3][lane] == 0 && x > ex)) {
          W.e[0][lane] = (u32)x;
          W.e[1][lane] = (u32)(x >> 32);
          W.e[2][lane] = 0;
          W.e[3][lane] = 0;
          evalid = true;
        }
      };
      // a finish that may change a maximum or is an error; every other finish only frees the lane
      auto finish = [&]() {
        if (st > ST_CAP) {
          atomicOr(&A.recs[req].errors, ERR_ITER_CAP);
          atomicAdd(&A.recs[req].failures, 1ull);
          return;
        }
        // the seed fell below its start inside the last even run; st is an upper bound of sigma
        if (st >= thr_st) {
          // x = (vh:v), the value before that run.  i* = least i with x >> i < n: with
          // d = bitlen(x) - bitlen(n), i* is d when x >> d < n, else d + 1 (d <= b <= 31).
          const int d = (int)(vh ? 128u - __clzll(vh) : bitlen64(v)) - (int)bitlen64(n);
          u32 istar = 1;
          if (d >= 1) {
            const u64 ylo = (v >> d) | (vh << (64 - d)), yhi = vh >> d;
            istar = ((yhi == 0) & (ylo < n)) ? (u32)d : (u32)d + 1u;
          }
          st = st - b + istar;
          if (st >= thr_st) {
            W.c[0][lane] = st;
            pend |= 1u;
          }
        }
        if (evalid) {
          pend |= 2u;
          W.pe[0][lane] = W.e[0][lane];
          W.pe[1][lane] = W.e[1][lane];
          W.pe[2][lane] = W.e[2][lane];
          W.pe[3][lane] = W.e[3][lane];
        }
        if (pend) {
          W.c[1][lane] = (u32)n;
          W.c[2][lane] = (u32)(n >> 32);
          W.c[3][lane] = 0;
          W.c[4][lane] = req;
        }
      };
      // V: the 64-bit pair first, then one vote for every rare event of the step (a value at
      // or above 2^59, an excursion candidate, a finish that may offer); else a vote each,
      // the four-limb pair before the 64-bit one
      if (!V && __any_sync(FULL, slow)) {
        if (slow) slow_pair();
      }
      // 64-bit run pair (every lane computes it; active fast lanes keep the result): the
      // odd run (at most 7 steps) multiplies by less than 2^5, so the value stays below 2^64
      const bool fast = active & !slow & !jstep;
      const u32 a = ctz32((u32)v | 0x80u);
      const u64 x = (v >> a) * s_pow3[a] - 1;  // the value after the odd run
      const u32 bb = ctz32((u32)x | 0x80000000u);
      const u64 w = x >> bb;
      const u32 st2 = st + a + bb;
      // a run of bb = 0 leaves x, which exceeds the value before the odd run (>= n)
      const bool ff = fast & ((w < n) | (st2 > ST_CAP));
      const bool cand = fast & (x + 1 >= G);
      if (STATS && fast) {
        X.pairs++;
        X.fast++;
      }
      if (fast) {
        st = st2;
        b = bb;
        fin = ff;
        v = ff ? x : w + 1;  // the finish reads the value before the even run
      }
      if (V) {
        const bool rare = slow | cand | (fin & ((st > ST_CAP) | (st >= thr_st) | evalid));
        if (__any_sync(FULL, rare)) {
          if (slow) slow_pair();
          if (cand) take_candidate(x);
          if (fin & ((st > ST_CAP) | (st >= thr_st) | evalid)) finish();
        }
      } else {
        if (__any_sync(FULL, cand)) {
          if (cand) take_candidate(x);
        }
        const bool need = fin & ((st > ST_CAP) | (st >= thr_st) | evalid);
        if (__any_sync(FULL, need)) {
          if (need) finish();
        }
      }
      active = active & !fin;
    }
  }
  if (STATS && A.stats) {
    if (lane == 0) {
      atomicAdd(&A.stats[8], t_offer);
      atomicAdd(&A.stats[9], t_refill);
      atomicAdd(&A.stats[10], t_lanes);
    }
    // [11], [12]: run pairs taken and seeds finished at expansion
    // run pairs, excursion slow paths, replays, jumps, pops, expansions, passes, offers,
    // table steps [13], windows [14], 64-bit pairs [15]
    const u32 c[13] = {X.pairs, X.slow_e, X.replay, X.jump, X.pop,  X.exp,   X.pass,
                       X.offer, X.tab,    X.win,    X.fast, X.xpairs, X.xfin};
    const u32 slot[13] = {0, 1, 2, 3, 4, 5, 6, 7, 13, 14, 15, 11, 12};
#pragma unroll
    for (int i = 0; i < 13; i++) {
      u32 x = c[i];
      if (i == 5 || i == 6) x = (lane == 0) ? x : 0u;  // warp-uniform counters
#pragma unroll
      for (u32 d = 16; d; d >>= 1) x += __shfl_xor_sync(FULL, x, d);
      if (lane == 0) atomicAdd(&A.stats[slot[i]], (ull)x);
    }
  }
  if (lane == 0 && w_req != 0xFFFFFFFFu) {
    if (W.acc_seeds) atomicAdd(&A.recs[w_req].seeds, W.acc_seeds);
    atomicAdd(&A.recs[w_req].items_done, W.acc_items);
  }
  cp_async_wait_all();
}

// ------------------------------------------------------------------
// Launchers.
// ------------------------------------------------------------------
constexpr size_t RANGE64_SMEM = sizeof(Warp64) * R64_WARPS;

// (run pairs per pass R, minimum resident blocks per SM, in-loop table steps J, expansion
// window length JW, windows per seed C, run pairs per seed at expansion M, then M2 more for
// the seeds the first M left running, packed into lanes; V: one vote per run-loop step for
// every rare event; PT: after the first step of a pass, idle lanes take queued seeds only
// when at least PT of them are idle; NQ: the k-step jump multiplies a block number q below
// 2^32 with two wide multiply-adds).  Measured on B200, 2^36 seeds at 2^40 with k = 24
// (2^34 at 2^47; the 2^38 block at 2^40), best of three, side by side in one process:
// 11.11 ms (3.07; 43.54) for variant 0, 11.09 (3.02; 43.60) for 1, 11.25 (3.09; 44.15) for
// 2 (the previous default: a pop at every step), 11.14 (3.06; 43.72) for 3, 11.18 (3.04;
// 43.90) for 6; pop thresholds of 8, 16 and 24 gave 43.57, 43.55 and 43.54 ms on the block.
// Earlier, with PT = 1 and no NQ: 11.60 (3.18) for 4, 11.77 (3.18) for 5 (the form without
// the second stage or the single vote), 11.97 (3.23) for 7; 3 + 3 + 3 pairs in three stages
// took 12.06 ms, 2 + 4 took 12.21, and the lanes' two entries stepped in lockstep 12.15.
#define CZ_RANGE64_VARIANTS(X)                                                                                   \
  X(0, 2, 4, 0, 11, 1, 3, 4, true, 12, true) X(1, 2, 4, 0, 10, 1, 3, 4, true, 12, true)                          \
  X(2, 2, 4, 0, 11, 1, 3, 4, true, 1, false) X(3, 2, 4, 0, 11, 1, 3, 5, true, 12, true)                          \
  X(4, 2, 4, 0, 11, 1, 5, 0, true, 1, false) X(5, 2, 4, 0, 11, 1, 5, 0, false, 1, false)                         \
  X(6, 2, 4, 0, 11, 1, 3, 4, true, 33, false) X(7, 2, 3, 0, 11, 1, 3, 4, true, 1, false)

int range64_variants() { return 8; }

// FNV-1a of the variant table's parameters: part of the autotuner's cache key, so that a
// choice cached for another table is not applied to this one.
uint32_t range64_variant_rev() {
  static const int p[] = {
#define X(id, rm, mb, j, jw, cw, m, m2, vo, pt, nq) id, rm, mb, j, jw, cw, m, m2, (int)(vo), pt, (int)(nq),
      CZ_RANGE64_VARIANTS(X)
#undef X
  };
  uint32_t h = 2166136261u;
  for (int x : p) h = (h ^ (uint32_t)x) * 16777619u;
  return h;
}

uint32_t range64_max_seed_bits() { return SEED_BITS_64; }

cudaError_t launch_range64(const RangeArgs& a, int variant, u32 grid, cudaStream_t st) {
  if (a.negative || a.seed_bits > SEED_BITS_64) return cudaErrorInvalidValue;
  switch (variant) {
#define X(id, rm, mb, j, jw, cw, m, m2, vo, pt, nq)                                                         \
  case id:                                                                       \
    k_range64<rm, mb, j, jw, cw, m, m2, vo, pt, nq, false><<<grid, R64_WARPS * 32, RANGE64_SMEM, st>>>(a);  \
    break;
    CZ_RANGE64_VARIANTS(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_range64_stats(const RangeArgs& a, int variant, u32 grid, cudaStream_t st) {
  if (a.negative || a.seed_bits > SEED_BITS_64) return cudaErrorInvalidValue;
  switch (variant) {
#define X(id, rm, mb, j, jw, cw, m, m2, vo, pt, nq)                                                        \
  case id:                                                                      \
    k_range64<rm, mb, j, jw, cw, m, m2, vo, pt, nq, true><<<grid, R64_WARPS * 32, RANGE64_SMEM, st>>>(a);  \
    break;
    CZ_RANGE64_VARIANTS(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t range64_occupancy(int variant, int* bps) {
  switch (variant) {
#define X(id, rm, mb, j, jw, cw, m, m2, vo, pt, nq) \
  case id:               \
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_range64<rm, mb, j, jw, cw, m, m2, vo, pt, nq, false>, R64_WARPS * 32, RANGE64_SMEM);
    CZ_RANGE64_VARIANTS(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
}

// Opts every 64-bit range kernel into RANGE64_SMEM of dynamic shared memory.
cudaError_t range64_init() {
  cudaError_t e = cudaSuccess;
#define X(id, rm, mb, j, jw, cw, m, m2, vo, pt, nq)                                                                                            \
  if (e == cudaSuccess)                                                                                             \
    e = cudaFuncSetAttribute(k_range64<rm, mb, j, jw, cw, m, m2, vo, pt, nq, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,              \
                             (int)RANGE64_SMEM);                                                                    \
  if (e == cudaSuccess)                                                                                             \
    e = cudaFuncSetAttribute(k_range64<rm, mb, j, jw, cw, m, m2, vo, pt, nq, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,               \
                             (int)RANGE64_SMEM);
  CZ_RANGE64_VARIANTS(X)
#undef X
  return e;
}

}  // namespace cz
