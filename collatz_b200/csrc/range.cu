// range.cu -- range verification: every seed n of [offset, offset+size)
// that survives the 2^k residue sieve and the mod-9 sieve is iterated
// until it falls below its start; outputs are the seeds checked, the
// maximum stopping time and the maximum excursion (each with the smallest
// seed on ties) and the seeds that did not finish.
//
// One kernel serves the plain single range and the batched form: the
// host lowers every request into segments of work items, and persistent
// warps claim items from a global cursor.  A sieved item is 64 consecutive
// entries of one mod-9 class of the (class-major) survivor table for one
// block q (seeds n = q 2^k + r); the warp stages them with cp.async, sets
// every seed up with a warp scan into its shared-memory queue, and idle
// lanes pull seeds from the queue with one ballot per step.  A seed starts
// after one k-step jump, T^k(n) + 1 = q 3^f + c (no descent is possible in
// those k steps), and, when bit lengths prove it exact, 8 more steps from a
// 256-entry shared-memory table.  It then runs odd/even runs in 4 x 32-bit
// limbs -- or on one 64-bit value while the warp's values are below 2^59 --
// with the exact stopping time and excursion.  A value that could leave
// 2^128 sends the seed to the widen list, re-run from scratch with 6 and then
// 8 limbs.  Before the kernel, threshold scouts run the first seeds of each
// request in full to give its prefilter keys a head start.
#include <cuda_runtime.h>

#include "range_shared.cuh"

namespace cz {

constexpr u32 RWARPS = 7;  // warps per block of k_range

// Per-warp state in shared memory.  Queue entries are fully set-up seeds:
// qa = v = T^s(n) + 1, qb = (n0, n1, n2, meta) with meta [7:0] steps s,
// [12:8] item slot, [13] v - 1 is an excursion candidate, [23:16] bitlen(n).
struct RangeWarp {
  uint4 qa[RQ];
  uint4 qb[RQ];
  uint4 ring[RR];          // per item slot: request, sigma threshold, excursion window (lo, hi)
  u32 ring_end[RR];        // per item slot: queue position after the item's last seed
  uint4 stage[RANGE_ITEM]; // survivor entries of the staged item (cp.async)
  u32 e[4][32];            // per lane: seed-local max excursion
  u32 pe[4][32];           // per lane: excursion of a pending offer
  u32 c[5][32];            // per lane: pending offer [0] sigma [1..3] seed [4] request
  u32 bln[32];             // per lane: bit length of the seed
  RangeSeg seg;            // cached segment
  StagedItem nxt;
  ull item, claim_hi, seg_lo, seg_hi, qi, acc_seeds, acc_items;
  u32 chunk, since_thr, ring_seq, thr_bl, head, pad;
};

// Diagnostics of the stats variant: cycles waiting for staged entries,
// staging the next item and refreshing thresholds; items expanded, seeds
// set up by the k-step jump and by an exact replay of the first k steps.
struct ExpandStats {
  ull t_wait = 0, t_stage = 0, t_thr = 0, t_sub = 0;
  u32 c_exp = 0, c_jump = 0, c_replay = 0, c_win = 0;
};

// Expands the staged item into the warp's seed queue (W.qa, W.qb from
// position tail): waits for its entries, starts staging the next item,
// refreshes the request's thresholds when the request changes (and every 64
// items), applies the mod-9 sieve when the segment asks for it, ranks the
// seeds with a warp scan and writes each seed's start state -- the k-step
// jump v = q 3^f + c, or n + 1 when the excursion threshold could be
// reached within the first k steps -- with its item slot.  Sets exhausted
// when no item is left.  Returns false, doing nothing, while the item slot
// it would take still has seeds in the queue (queued seeds read their
// request and thresholds from their item's slot when they are popped, so a
// slot is reused only after the last seed of its previous item has left the
// queue; the queue is then not empty).  Warp-uniform.
// Up to M run pairs of a seed at expansion on four limbs, with every lane
// busy.  A pair is kept only in the common case: the value stays below 2^114
// before the odd run (so it stays below 2^119 after it), the value after the
// odd run is below the excursion gate window, and the seed either does not
// descend or descends with a stopping time below thr_st.  Otherwise the pair
// is left to the run loop.  Returns false when the seed finished here.
template <int M>
__device__ __forceinline__ bool first_pairs4(u32& V0, u32& V1, u32& V2, u32& V3, u32& s0, u32 n0, u32 n1, u32 n2,
                                             u64 gate_w, u32 thr_st) {
#pragma unroll
  for (int m = 0; m < M; m++) {
    if (V3 >= (1u << 18)) break;
    u32 y0 = V0, y1 = V1, y2 = V2, y3 = V3;
    const u32 a = ctz32(y0 | 0x80u);
    odd_run4(y0, y1, y2, y3, a, pow3_le7(a));
    if (!lt96c(y1, y2, y3, (u32)gate_w, (u32)(gate_w >> 32), 0u)) break;  // candidate: the loop takes it
    y0 -= 1;  // y0 == 0 gives b == 0 below, and the borrow cancels against the +1
    const u32 b = ctz32(y0 | 0x80000000u);
    const u32 w0 = __funnelshift_r(y0, y1, b), w1 = __funnelshift_r(y1, y2, b);
    const u32 w2 = __funnelshift_r(y2, y3, b), w3 = y3 >> b;
    const u32 st2 = s0 + a + b;
    if ((w3 == 0) & (b != 0) & lt96c(w0, w1, w2, n0, n1, n2)) {
      if (st2 >= thr_st) break;  // sigma may reach the maximum: the loop takes it
      return false;
    }
    V0 = w0 + 1;
    V1 = w1;
    V2 = w2;
    V3 = w3;
    add_carry3(V1, V2, V3, (V0 == 0) & (b != 0));
    s0 = st2;
  }
  return true;
}

template <bool STATS, bool NEG, int JW, int M, class WT>
__device__ __forceinline__ bool expand_one(WT& W, const RangeArgs& A, const uint4* __restrict__ T, u32 lane, u32 k,
                                           u32 k9, const unsigned long long* s_p3, const u32* s_win, u32 head,
                                           u32& tail, bool& exhausted, u32& w_thr_st, u32& w_req, u64& w_gate,
                                           ExpandStats& X) {
  if ((int)(W.ring_end[W.ring_seq & (RR - 1)] - head) > 0) return false;
  if (STATS) X.t_sub = clock64();
  cp_async_wait_all();  // this lane's copies of the staged item
  __syncwarp();
  if (STATS) {
    const ull now = clock64();
    X.t_wait += now - X.t_sub;
    X.t_sub = now;
  }
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
  if (STATS) {
    const ull now = clock64();
    X.t_stage += now - X.t_sub;
    X.t_sub = now;
  }
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
  if (STATS) {
    const ull now = clock64();
    X.t_thr += now - X.t_sub;
    X.t_sub = now;
  }
  const u32 w_thr_bl = W.thr_bl;
  const u64 gate_w = w_gate;
  const u32 slot = W.ring_seq & (RR - 1);
  u32 mask = 0, total, seeds;
  u32 pos;
  if (it.kind == 0) {
    const u32 q0 = (u32)it.q_lo, q1 = (u32)(it.q_lo >> 32), q2 = it.q_hi;
    // per item (warp-uniform): n = q 2^k | r as limbs (k <= 34), bitlen(n) = bitlen(q) + k
    const u32 kb = k & 31;
    const u32 t0 = q0 << kb, t1 = __funnelshift_l(q0, q1, kb), t2 = __funnelshift_l(q1, q2, kb);
    const u32 qk0 = (k >= 32) ? 0u : t0, qk1 = (k >= 32) ? t0 : t1, qk2 = (k >= 32) ? t1 : t2;
    const u32 nbl = (q2 ? 96u - __clz(q2) : (q1 ? 64u - __clz(q1) : 32u - __clz(q0))) + k;
    const u32 meta_item = (slot << 8) | (nbl << 16);
    const bool jump_ok_base = true;
    if (it.mod9) {  // segments of whole kept classes (the usual case) need no per-entry test
      const u32 b9 = (mod9_96(q0, q1, q2) * k9) % 9u;
#pragma unroll
      for (u32 j = 0; j < RANGE_ITEM / 32; j++) {
        if (it.sbase + j * 32 + lane < it.send) {
          u32 x = b9 + ((e[j].y >> 16) & 0xFFu);
          x = (x >= 9u) ? x - 9u : x;
          if (((NEG ? KEEP9N : KEEP9) >> x) & 1u) mask |= 1u << j;
        }
      }
    } else {
#pragma unroll
      for (u32 j = 0; j < RANGE_ITEM / 32; j++)
        if (it.sbase + j * 32 + lane < it.send) mask |= 1u << j;
    }
    // each entry in turn: its seed's start state, then one ballot places the lanes' seeds
    seeds = __reduce_add_sync(FULL, __popc(mask));
    total = 0;
#pragma unroll
    for (u32 j = 0; j < RANGE_ITEM / 32; j++) {
      bool keep = false;
      u32 V0 = 0, V1 = 0, V2 = 0, V3 = 0, s0 = 0, m0 = 0, m1 = 0;
      if ((mask >> j) & 1u) {
        const u32 f = (e[j].y >> 8) & 0xFFu, emax = e[j].y >> 24;
        m0 = qk0 | e[j].x;
        m1 = qk1 | (e[j].y & 0xFFu);
        // T^0..T^k(n) < 2^emax (n + 1 + k) <= 2^(bitlen(n) + 1 + emax): skip them when that is
        // below the excursion threshold, else replay the first k steps exactly
        if (jump_ok_base && nbl + 1 + emax < w_thr_bl) {
          // v = q 3^f + c in 32-bit limbs (3^f < 2^64, c < 2^64)
          const u64 p = s_p3[f];
          const u32 p0 = (u32)p, p1 = (u32)(p >> 32);
          const u64 a = (u64)q0 * p0 + e[j].z;
          const u64 bb = (u64)q0 * p1 + (a >> 32) + e[j].w;
          const u64 cc = (u64)q1 * p0 + (u32)bb;
          const u64 dd = (u64)q1 * p1 + (bb >> 32) + (cc >> 32);
          V0 = (u32)a;
          V1 = (u32)cc;
          V2 = (u32)dd;
          V3 = (u32)(dd >> 32);
          if (q2) {  // q >= 2^64 (seeds >= 2^(64+k))
            const u64 ee = (u64)q2 * p0 + V2;
            V2 = (u32)ee;
            V3 += q2 * p1 + (u32)(ee >> 32);
          }
          s0 = k;
          if (JW && !NEG) {
            // JW more steps at once when they can neither descend nor reach the
            // excursion threshold: x = T^k(n) = a 2^JW + r gives T^i(x) = a 2^(JW-i) 3^f_i +
            // T^i(r) for i <= JW, so a g(r) <= T^i(x) < (a + 1) h(r) (g, h: the least and
            // largest 2^(JW-i) 3^f_i); bit lengths test both bounds
            const u32 x0 = V0 - 1, x1 = V1 - (V0 == 0), x2 = V2 - ((V0 | V1) == 0), x3 = V3 - ((V0 | V1 | V2) == 0);
            const u32 te = s_win[x0 & ((1u << JW) - 1u)];
            const u32 xb = x3 ? 128u - __clz(x3) : (x2 ? 96u - __clz(x2) : (x1 ? 64u - __clz(x1) : 32u - __clz(x0)));
            const u32 glen = (te >> 22) & 31u, hlen = te >> 27;
            if ((xb + glen >= nbl + (u32)JW + 2u) & (xb + hlen < w_thr_bl + (u32)JW) & (xb <= 100u)) {
              u32 y0 = x0, y1 = x1, y2 = x2, y3 = x3;
              odd_run4(y0, y1, y2, y3, (u32)JW, (u32)s_p3[(te >> 18) & 15u]);  // (x >> JW) 3^f_JW
              // + T^JW(r) + 1 (back to v space)
              asm("add.cc.u32 %0, %0, %4;\n\t"
                  "addc.cc.u32 %1, %1, 0;\n\t"
                  "addc.cc.u32 %2, %2, 0;\n\t"
                  "addc.u32 %3, %3, 0;"
                  : "+r"(y0), "+r"(y1), "+r"(y2), "+r"(y3)
                  : "r"((te & 0x3FFFFu) + 1u));
              V0 = y0;
              V1 = y1;
              V2 = y2;
              V3 = y3;
              s0 = k + (u32)JW;
              if (STATS) X.c_win++;
            }
          }
          if (STATS) X.c_jump++;
        } else {
          if (NEG) {  // u = n - 1 (n >= 2^k: no borrow out of 96 bits)
            V0 = m0 - 1;
            V1 = m1 - (m0 == 0);
            V2 = qk2 - ((m0 | m1) == 0);
            V3 = 0;
          } else {
            V0 = m0 + 1;
            V1 = m1 + (V0 == 0);
            V2 = qk2 + ((V0 | V1) == 0);
            V3 = (V0 | V1 | V2) == 0;
          }
          s0 = 0;
          if (STATS) X.c_replay++;
        }
        keep = true;
        if (M > 0 && !NEG) keep = first_pairs4<M>(V0, V1, V2, V3, s0, m0, m1, qk2, gate_w, w_thr_st);
      }
      const u32 bk = __ballot_sync(FULL, keep);
      if (keep) {
        // excursion candidate T^s(n) = v - 1 <= v: bits 32..95 of v against the threshold
        // T': the candidate is u + 1, whose window exceeds u's by at most 1
        const u32 cand =
            ((V3 != 0) | ((((u64)V2 << 32) | V1) >= (NEG ? gate_w - (gate_w != 0) : gate_w))) ? 1u : 0u;
        const u32 at = (tail + total + __popc(bk & lanemask_lt())) & (RQ - 1);
        W.qa[at] = make_uint4(V0, V1, V2, V3);
        W.qb[at] = make_uint4(m0, m1, qk2, s0 | meta_item | (cand << 13));
      }
      total += __popc(bk);
    }
  } else {
    // integers below 2^k: [d, d + 64) of [q_lo, d_hi), no residue sieve
    const ull d = it.q_lo + 2ull * lane;
#pragma unroll
    for (u32 j = 0; j < 2; j++) {
      const ull n = d + j;
      const u32 r9 = (u32)(n % 9u);
      const bool keep9 = NEG ? ((((KEEP9N >> r9) & 1u) != 0) | (n == 5)) : (((KEEP9 >> r9) & 1u) != 0);
      if (n < it.d_hi && n >= 2 && (!it.mod9 || keep9)) mask |= 1u << j;
    }
    pos = tail + warp_excl_scan(__popc(mask), &total);
    seeds = total;
#pragma unroll
    for (u32 j = 0; j < 2; j++) {
      if ((mask >> j) & 1u) {
        const ull n = d + j;
        const u32 nbl = 64u - __clzll(n);
        const u32 cand = ((n >> 32) >= gate_w) ? 1u : 0u;
        const ull v = NEG ? n - 1 : n + 1;
        W.qa[pos & (RQ - 1)] = make_uint4((u32)v, (u32)(v >> 32), 0u, 0u);
        W.qb[pos & (RQ - 1)] = make_uint4((u32)n, (u32)(n >> 32), 0u, (slot << 8) | (cand << 13) | (nbl << 16));
        pos++;
      }
    }
  }
  __syncwarp();
  if (lane == 0) {
    W.ring[slot] = make_uint4(rq, w_thr_st, (u32)w_gate, (u32)(w_gate >> 32));
    W.ring_end[slot] = tail + total;
    W.ring_seq++;
    W.acc_seeds += seeds;
    W.acc_items++;
  }
  if (STATS) X.c_exp++;
  tail += total;
  __syncwarp();
  return true;
}

// Offers of several pending lanes (all lanes call this together): a value that
// another pending lane of the same request beats -- larger, or equal with a
// smaller seed -- cannot be the request's maximum, so its bit is dropped and
// only the best of each request is offered.  Kept out of line: it runs in few
// passes, and inlined it costs the lane loop registers.
__device__ __noinline__ u32 drop_dominated(RangeWarp& W, u32 lane, u32 pend, u32 pm) {
  const u32 m1 = __ballot_sync(FULL, pend & 1u), m2 = __ballot_sync(FULL, pend & 2u);
  __syncwarp();
  if (pend) {
    const u32 rq = W.c[4][lane], s0 = W.c[1][lane], s1 = W.c[2][lane], s2 = W.c[3][lane];
    for (u32 m = pm & ~(1u << lane); m; m &= m - 1) {
      const u32 j = __ffs(m) - 1;
      if (W.c[4][j] != rq) continue;
      const u32 t0 = W.c[1][j], t1 = W.c[2][j], t2 = W.c[3][j];
      const bool j_smaller = (t2 != s2) ? (t2 < s2) : ((t1 != s1) ? (t1 < s1) : (t0 < s0));
      if ((pend & 1u) && ((m1 >> j) & 1u)) {
        const u32 sj = W.c[0][j], si = W.c[0][lane];
        if (sj > si || (sj == si && j_smaller)) pend &= ~1u;
      }
      if ((pend & 2u) && ((m2 >> j) & 1u)) {
        int c = 0;  // E_j against this lane's E, from the top limb
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

template <int R, int MINB, bool STATS = false, bool NEG = false, int JW = 0, bool N64 = false, int M = 0>
__global__ void __launch_bounds__(RWARPS * 32, MINB) k_range(const RangeArgs A) {
  // diagnostics (STATS variant only): run pairs, excursion slow paths, replays, jumps, pops,
  // expansions, passes, offers; clock64 cycles per phase (lane 0)
  u32 c_iter = 0, c_slow = 0, c_pop = 0, c_blk = 0, c_offer = 0, c_narrow = 0;
  ull t_offer = 0, t_refill = 0, t_lanes = 0, t_mark = 0;
  ExpandStats X;
  extern __shared__ __align__(16) unsigned char range_smem[];
  RangeWarp* S = reinterpret_cast<RangeWarp*>(range_smem);
  __shared__ unsigned long long s_p3[41];
  __shared__ u32 s_pow3[9], s_keep9[9];
  __shared__ u32 s_win[JW ? (1u << JW) : 1];  // the JW-step table (build_step_table)
  if (JW) build_step_table(s_win, (u32)JW);
  const u32 lane = lane_id();
  RangeWarp& W = S[threadIdx.x >> 5];
  if (threadIdx.x < 41) {
    unsigned long long p = 1;
    for (u32 i = 0; i < threadIdx.x; i++) p *= 3;
    s_p3[threadIdx.x] = p;
    if (threadIdx.x < 9) s_pow3[threadIdx.x] = (u32)p;
  }
  if (threadIdx.x >= 64 && threadIdx.x < 73) {
    const u32 r = threadIdx.x - 64;  // bit j: (r + j) mod 9 survives
    u32 m = 0;
    for (u32 j = 0; j < 32; j++) m |= ((KEEP9 >> ((r + j) % 9u)) & 1u) << j;
    s_keep9[r] = m;
  }
  if (lane == 0) {
    W.item = ~0ull;
    W.claim_hi = 0;
    W.seg_lo = 1;
    W.seg_hi = 0;
    W.qi = W.acc_seeds = W.acc_items = 0;
    W.chunk = W.since_thr = W.ring_seq = W.thr_bl = W.head = 0;
    W.nxt.valid = 0;
  }
  W.ring_end[lane] = 0;  // RR == 32: one slot per lane
  __syncthreads();

  const u32 k = A.k;
  const u32 k9 = (u32)((1ull << (k % 6)) % 9ull);  // 2^k mod 9 (2^6 = 1 mod 9)
  const uint4* __restrict__ T = reinterpret_cast<const uint4*>(A.table);
  stage_next(W, W.stage, A, T, lane);

  // ---- warp-uniform state (the rest lives in W) ----
  u32 head = 0, tail = 0;  // queued seeds [head, tail)
  bool exhausted = false;
  u32 w_thr_st = 0, w_req = 0xFFFFFFFFu;
  u64 w_gate = 0;  // excursion threshold, bits 32..95 (all ones when it is >= 2^96)
  // ---- lane state ----
  u32 v0 = 0, v1 = 0, v2 = 0, v3 = 0, n0 = 0, n1 = 0, n2 = 0, st = 0, req = 0, thr_st = 0;
  u64 gate = 0;  // the lane's excursion threshold window (bits 32..95)
  bool active = false, evalid = false;
  u32 pend = 0;

#define POP_NEXT(idx_)                                                               \
  do {                                                                               \
    if (idx_ < tail) {                                                               \
      const uint4 a_ = W.qa[idx_ & (RQ - 1)], b_ = W.qb[idx_ & (RQ - 1)];            \
      v0 = a_.x;                                                                     \
      v1 = a_.y;                                                                     \
      v2 = a_.z;                                                                     \
      v3 = a_.w;                                                                     \
      n0 = b_.x;                                                                     \
      n1 = b_.y;                                                                     \
      n2 = b_.z;                                                                     \
      st = b_.w & 0xFFu;                                                             \
      const uint4 g_ = W.ring[(b_.w >> 8) & 31u];                                    \
      req = g_.x;                                                                    \
      W.bln[lane] = (b_.w >> 16) & 0xFFu;                                            \
      if (g_.x == w_req) { /* the warp's thresholds are the freshest */              \
        thr_st = w_thr_st;                                                           \
        gate = w_gate;                                                               \
      } else {                                                                       \
        thr_st = g_.y;                                                               \
        gate = ((u64)g_.w << 32) | g_.z;                                             \
      }                                                                              \
      evalid = (b_.w >> 13) & 1u;                                                    \
      if (evalid) { /* the value T^s(n) = v -/+ 1 is an excursion candidate */        \
        u32 x_[4];                                                                   \
        value_of<NEG>(v0, v1, v2, v3, x_);                                           \
        W.e[0][lane] = x_[0];                                                        \
        W.e[1][lane] = x_[1];                                                        \
        W.e[2][lane] = x_[2];                                                        \
        W.e[3][lane] = x_[3];                                                        \
      }                                                                              \
      active = true;                                                                 \
      if (STATS) c_pop++;                                                            \
      if (v3 >= OVF3) { /* the jump already left 2^119 */                            \
        widen_seed(A, req, n0, n1, n2);                                              \
        active = false;                                                              \
      }                                                                              \
    }                                                                                \
  } while (0)

// The value T^s(n) = v -/+ 1 at or above the excursion threshold window: keep
// it as the seed's maximum when it is the largest so far.
#define EXC_CANDIDATE()                                                                  \
  do {                                                                                   \
    if (STATS) c_slow++;                                                                 \
    u32 xv_[4];                                                                          \
    value_of<NEG>(v0, v1, v2, v3, xv_);                                                  \
    bool take_ = !evalid;                                                                \
    if (evalid)                                                                          \
      take_ = lt96c(W.e[0][lane], W.e[1][lane], W.e[2][lane], xv_[0], xv_[1], xv_[2])    \
                  ? (W.e[3][lane] <= xv_[3])                                             \
                  : (W.e[3][lane] < xv_[3]);                                             \
    if (take_) {                                                                         \
      W.e[0][lane] = xv_[0];                                                             \
      W.e[1][lane] = xv_[1];                                                             \
      W.e[2][lane] = xv_[2];                                                             \
      W.e[3][lane] = xv_[3];                                                             \
      evalid = true;                                                                     \
    }                                                                                    \
  } while (0)

  if (STATS) t_mark = clock64();
  for (;;) {
    if (STATS) {
      c_blk++;
      const ull now = clock64();
      t_lanes += now - t_mark;
      t_mark = now;
    }
    // ---- warp-synchronous part: offers of finished seeds (rare), refill, exit ----
    u32 pm = __ballot_sync(FULL, pend != 0);
    if (pm) {  // offers (rare)
      if (pm & (pm - 1)) {
        // several pending lanes (a warp's first seeds all finish under zero thresholds):
        // offer only the best of each request
        pend = drop_dominated(W, lane, pend, pm);
        pm = __ballot_sync(FULL, pend != 0);
      }
      while (pm) {
        const u32 leader = __ffs(pm) - 1;
        const u32 lp = __shfl_sync(FULL, pend, leader), lreq = W.c[4][leader];
        if (lane == leader) {
          const u32 seed[4] = {W.c[1][lane], W.c[2][lane], W.c[3][lane], 0};
          if (STATS) c_offer++;
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
    // ---- refill: keep 32 R seeds queued (each lane pops at most R per pass) ----
    while (tail - head < 32u * R && !exhausted) {
      if (!expand_one<STATS, NEG, JW, M>(W, A, T, lane, k, k9, s_p3, s_win, head, tail, exhausted, w_thr_st, w_req,
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

    // ---- lanes: R times (take a seed if idle, one odd run and one even run) ----
#pragma unroll
    for (int r = 0; r < R; r++) {
      {
        // idle lanes take the next queued seeds (a pending offer keeps its scratch until the next pass)
        const u32 want = __ballot_sync(FULL, !active && !pend);
        if (want) {
          const u32 take = min((u32)__popc(want), tail - head);
          if (!active && !pend) {
            const u32 rank = __popc(want & lanemask_lt());
            if (rank < take) POP_NEXT(head + rank);
          }
          head += take;
        }
      }
      // 64-bit body while every active lane's value is below 2^59: an odd run of at most 7
      // steps multiplies by less than 2^5, so the value stays below 2^64 (a warp-uniform
      // choice made again at every step; the 128-bit body below is the general one)
      const bool narrow = N64 && !NEG && __all_sync(FULL, !active || (((v2 | v3) == 0) & (v1 < (1u << 27))));
      if (!active) continue;
      u32 b;
      bool fin;
      if (N64 && !NEG && narrow) {
        u64 v = ((u64)v1 << 32) | v0;
        const u32 a = ctz32(v0 | (1u << 7));
        v = (v >> a) * s_pow3[a];  // shared table: the load/store pipe, not the busy ALU pipe
        st += a;
        if (STATS) {
          c_iter++;
          c_narrow++;
        }
        v0 = (u32)v;
        v1 = (u32)(v >> 32);
        if ((v >> 32) >= gate) EXC_CANDIDATE();  // v2 = v3 = 0
        const u64 x = v - 1;
        b = ctz32((u32)x | 0x80000000u);
        const u64 w = x >> b;
        st += b;
        fin = ((b != 0) & ((n2 != 0) | (w < (((u64)n1 << 32) | n0)))) | (st > ST_CAP);
        const u64 y = fin ? x : w + 1;  // the finish reads v - 1; else the next state w + 1
        v0 = (u32)y;
        v1 = (u32)(y >> 32);
      } else {
        {
          // odd run capped at 7 steps (a longer run continues in the next pass, after an empty
          // even run)
          const u32 a = ctz32(v0 | (1u << 7));
          // 3^a: the shared table where this body is the hot one (measured: the
          // frontier's four-limb kernel gains 1 %), register lookups beside the
          // 64-bit body (the table there cost the block 0.5 %)
          odd_run4(v0, v1, v2, v3, a, N64 ? pow3_le7(a) : s_pow3[a]);
          st += a;
          if (STATS) c_iter++;
        }
        // excursion / overflow gate: (v3:v2:v1) >= (0:gate) (T': >= gate - 1, since the
        // value v + 1 has a window at most 1 above v's)
        const u64 g_eff = NEG ? gate - (gate != 0) : gate;
        if (!lt96c(v1, v2, v3, (u32)g_eff, (u32)(g_eff >> 32), 0u)) {
          if (v3 >= OVF3) {
            // the next odd run could leave 128 bits: re-run this seed with wider limbs
            widen_seed(A, req, n0, n1, n2);
            active = false;
            continue;
          }
          EXC_CANDIDATE();  // bits 32..95 at or above the threshold
        }
        if (NEG) {
          // t = u + 1 with a full carry (a low limb of all ones gives b = 31 below)
          v0 += 1;
          add_carry3(v1, v2, v3, v0 == 0);
        } else {
          v0 -= 1;  // v0 == 0 gives b == 0 below, and the borrow cancels against the +1
        }
        b = ctz32(v0 | 0x80000000u);
        const u32 w0 = __funnelshift_r(v0, v1, b), w1 = __funnelshift_r(v1, v2, b);
        const u32 w2 = __funnelshift_r(v2, v3, b), w3 = v3 >> b;
        st += b;
        fin = ((w3 == 0) & (b != 0) & lt96c(w0, w1, w2, n0, n1, n2)) | (st > ST_CAP);
        if (fin) {
          // the finish below reads v (the value before the even run)
        } else if (NEG && (w3 == 0) & (w0 == n0) & (w1 == n1) & (w2 == n2)) {
          // T': back at the seed -- it lies on a cycle and never descends (the minima 5, 17)
          atomicAdd(&A.recs[req].failures, 1ull);
          active = false;
        } else if (NEG) {
          // u = w - 1 (w >= 1)
          v0 = w0 - 1;
          v1 = w1 - (w0 == 0);
          v2 = w2 - ((w0 | w1) == 0);
          v3 = w3 - ((w0 | w1 | w2) == 0);
        } else {
          v0 = w0 + 1;
          v1 = w1;
          v2 = w2;
          v3 = w3;
          add_carry3(v1, v2, v3, (v0 == 0) & (b != 0));
        }
      }
      if (fin) {
        if (st > ST_CAP) {
          atomicOr(&A.recs[req].errors, ERR_ITER_CAP);
          atomicAdd(&A.recs[req].failures, 1ull);
        } else {
          // the seed fell below its start inside this run; st is an upper bound of sigma
          if (st >= thr_st) {
            // i* = least i with (v-1) >> i < n.  With d = bitlen(v-1) - bitlen(n),
            // i* is d when (v-1) >> d < n, else d + 1.
            u32 t = v3, base = 96;
            if (!t) { t = v2; base = 64; }
            if (!t) { t = v1; base = 32; }
            if (!t) { t = v0; base = 0; }
            const int d = (int)(base + 32u - __clz(t)) - (int)W.bln[lane];
            u32 istar = 1;
            if (d >= 1) {
              const u32 y0 = __funnelshift_r(v0, v1, d), y1 = __funnelshift_r(v1, v2, d);
              const u32 y2 = __funnelshift_r(v2, v3, d), y3 = v3 >> d;
              istar = ((y3 == 0) & lt96c(y0, y1, y2, n0, n1, n2)) ? (u32)d : (u32)d + 1;
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
            W.c[1][lane] = n0;
            W.c[2][lane] = n1;
            W.c[3][lane] = n2;
            W.c[4][lane] = req;
          }
        }
        active = false;
        // a lane with a pending offer waits for the next pass (its scratch is in use)
      }
    }
  }
#undef EXC_CANDIDATE
#undef POP_NEXT
  if (STATS && A.stats && lane == 0) {
    atomicAdd(&A.stats[8], t_offer);
    atomicAdd(&A.stats[9], t_refill);
    atomicAdd(&A.stats[10], t_lanes);
    atomicAdd(&A.stats[11], X.t_wait);
    atomicAdd(&A.stats[12], X.t_stage);
    atomicAdd(&A.stats[13], X.t_thr);
  }
  if (STATS && A.stats) {
    u32 c[10] = {c_iter, c_slow, X.c_replay, X.c_jump, c_pop, X.c_exp, c_blk, c_offer, X.c_win, c_narrow};
#pragma unroll
    for (int i = 0; i < 10; i++) {
      u32 x = c[i];
      if (i == 5 || i == 6) x = (lane == 0) ? x : 0u;  // warp-uniform counters
#pragma unroll
      for (u32 d = 16; d; d >>= 1) x += __shfl_xor_sync(FULL, x, d);
      if (lane == 0) atomicAdd(&A.stats[i < 8 ? i : i + 6], (ull)x);  // windows, 64-bit pairs: [14], [15]
    }
  }
  if (lane == 0 && w_req != 0xFFFFFFFFu) {
    if (W.acc_seeds) atomicAdd(&A.recs[w_req].seeds, W.acc_seeds);
    atomicAdd(&A.recs[w_req].items_done, W.acc_items);
  }
  cp_async_wait_all();
}

// ------------------------------------------------------------------
// Wide re-run: one seed per thread with L limbs, from scratch.
// ------------------------------------------------------------------
template <int L, bool NEG>
__global__ void __launch_bounds__(128) k_range_wide(const WidenEntry* __restrict__ list, const u32* count,
                                                   u32 cap, ReqRec* recs, WidenEntry* next, u32 next_cap,
                                                   u32* next_count, u32 iter_cap) {
  const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  const u32 n = min(*count, cap);
  const u32 lane = lane_id();
  bool ok = false;
  WidenEntry e{0, 0, 0, 0};
  Limbs<L> v, N, E;
  unsigned long long st = 0;
  if (i < n) {
    e = list[i];
#pragma unroll
    for (int j = 0; j < L; j++) N.w[j] = (j == 0) ? e.n0 : (j == 1) ? e.n1 : (j == 2) ? e.n2 : 0u;
    v = N;
    if (NEG) dec_l<L>(v); else inc_l<L>(v);  // v = n + 1, or u = n - 1 for T'
    E = N;
    u32 it = 0;
    for (;;) {
      if (v.w[L - 1] >= (1u << 19) || ++it > iter_cap) {
        if (it > iter_cap) {
          atomicOr(&recs[e.req].errors, ERR_ITER_CAP);
          atomicAdd(&recs[e.req].failures, 1ull);
        } else if (next) {
          const u32 wi = atomicAdd(next_count, 1u);
          if (wi < next_cap) {
            next[wi] = e;
          } else {
            atomicOr(&recs[e.req].errors, ERR_WIDEN_FULL);
            atomicAdd(&recs[e.req].failures, 1ull);
          }
        } else {
          atomicAdd(&recs[e.req].failures, 1ull);
        }
        break;
      }
      const u32 a = ctz32(v.w[0] | (1u << 8));
      u32 m = 1;
      for (u32 j = 0; j < a; j++) m *= 3u;
      odd_run_l<L>(v, a, m);
      st += a;
      Limbs<L> x = v;  // the value: v - 1, or u + 1 for T'
      if (NEG) inc_l<L>(x); else dec_l<L>(x);
      if (limbs_lt<L>(E, x)) E = x;
      // even run on the value x
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
        st += s;
        ok = true;
        break;
      }
      st += b;
      if (NEG && !limbs_lt<L>(w, N) && !limbs_lt<L>(N, w)) {  // back at the seed: a cycle
        atomicAdd(&recs[e.req].failures, 1ull);
        break;
      }
      v = w;
      if (NEG) dec_l<L>(v); else inc_l<L>(v);
    }
  }
  u32 pm = __ballot_sync(FULL, ok);
  while (pm) {
    const u32 leader = __ffs(pm) - 1;
    if (lane == leader) {
      const u32 seed[4] = {e.n0, e.n1, e.n2, 0};
      rec_offer_st(recs + e.req, st, seed);
      rec_offer_e<L>(recs + e.req, E.w, seed);
    }
    pm &= pm - 1;
  }
}

// ------------------------------------------------------------------
// Threshold scouts, launched before k_range.  A request's prefilter keys
// start at zero, and the item cursor hands a small request's items to many
// warps at once, so without a head start most of its seeds would run under
// zero thresholds: replaying their first k steps, taking the excursion slow
// path at every odd run and offering at the end.  Lane j of warp i runs the
// j-th seed of request i's first work item in full (4 limbs), and the warp
// raises the request's keys to the largest stopping time and excursion among
// them.  These are seeds the request checks, so the keys stay lower bounds of
// its maxima, and k_range still offers them (values equal to a threshold pass
// every prefilter test).
// ------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_range_scout(const RangeArgs A, const u32* __restrict__ first_seg, u32 nreq) {
  const u32 wi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = lane_id();
  if (wi >= nreq) return;  // warp-uniform
  const u32 si = first_seg[wi];
  if (si >= A.nsegs) return;  // a request without seeds
  const RangeSeg g = A.segs[si];
  if (g.local0_lo | g.local0_hi) return;  // not the segment's first item
  // this lane's seed n (3 limbs): entry lane of the first item, or integer d_lo + lane
  bool have = false;
  Limbs<4> N;
  N.w[3] = 0;
  if (g.kind == 0) {
    const u32 idx = g.s_lo + lane;
    if (idx < g.s_hi && lane < RANGE_ITEM) {
      const RangeEntry e = A.table[idx];
      const u32 k = A.k, kb = k & 31;
      const u32 q0 = (u32)g.q_lo, q1 = (u32)(g.q_lo >> 32), q2 = g.q_hi;
      const u32 t0 = q0 << kb, t1 = __funnelshift_l(q0, q1, kb), t2 = __funnelshift_l(q1, q2, kb);
      N.w[0] = ((k >= 32) ? 0u : t0) | e.r_lo;
      N.w[1] = ((k >= 32) ? t0 : t1) | (e.meta & 0xFFu);
      N.w[2] = (k >= 32) ? t1 : t2;
      have = true;
      if (g.mod9) {
        const u32 k9 = (u32)((1ull << (k % 6)) % 9ull);
        u32 x = (mod9_96(q0, q1, q2) * k9) % 9u + ((e.meta >> 16) & 0xFFu);
        x = (x >= 9u) ? x - 9u : x;
        have = ((KEEP9 >> x) & 1u) != 0;
      }
    }
  } else {
    const ull n = g.q_lo + lane;
    if (n < g.d_hi && n >= 2 && (!g.mod9 || ((KEEP9 >> (u32)(n % 9u)) & 1u))) {
      N.w[0] = (u32)n;
      N.w[1] = (u32)(n >> 32);
      N.w[2] = 0;
      have = true;
    }
  }
  u32 sig = 0;
  ull ekey = 0;
  if (have) {
    Limbs<4> v = N, E = N;
    inc_l<4>(v);  // v = n + 1
    ull st = 0;
    for (u32 it = 0;; it++) {
      if (v.w[3] >= (1u << 19) || it > A.iter_cap) break;  // could leave 128 bits: no scout
      const u32 a = ctz32(v.w[0] | (1u << 8));
      odd_run_l<4>(v, a, pow3_le8(a));
      st += a;
      Limbs<4> x = v;
      dec_l<4>(x);
      if (limbs_lt<4>(E, x)) E = x;
      const u32 b = ctz32(x.w[0] | 0x80000000u);
      Limbs<4> w = x;
      shr_l<4>(w, b);
      if (b != 0 && limbs_lt<4>(w, N)) {
        u32 s = 1;
        for (; s < b; s++) {
          Limbs<4> y = x;
          shr_l<4>(y, s);
          if (limbs_lt<4>(y, N)) break;
        }
        sig = (u32)min(st + s, 0xFFFFFFFFull);
        ekey = key_of<4>(E.w);
        break;
      }
      st += b;
      v = w;
      inc_l<4>(v);
    }
  }
  sig = __reduce_max_sync(FULL, sig);
#pragma unroll
  for (u32 d = 16; d; d >>= 1) ekey = max(ekey, (ull)__shfl_xor_sync(FULL, ekey, d));
  if (lane == 0) {
    if (sig) atomicMax(&A.recs[g.req].st_key, (ull)sig);
    if (ekey) atomicMax(&A.recs[g.req].e_key, ekey);
  }
}

// ------------------------------------------------------------------
// Launchers.
// ------------------------------------------------------------------
int range_variants() { return 8; }

constexpr size_t RANGE_SMEM = sizeof(RangeWarp) * RWARPS;

cudaError_t launch_range_stats(const RangeArgs& a, u32 grid, cudaStream_t st) {
  k_range<2, 3, true, false, 8, false, 3><<<grid, RWARPS * 32, RANGE_SMEM, st>>>(a);
  return cudaGetLastError();
}

// (run pairs per pass, minimum resident blocks per SM, length JW of the jump-table window
// after the k-step jump (0: none), 64-bit body while the warp's values are below 2^59, run
// pairs per seed taken at expansion).  Measured on B200, 2^36 seeds at 2^60 + 3 2^34 with
// k = 34: 8.19 ms (variant 0), 8.43 (1), 10.13 (2), 9.08 (3), 9.63 (4), 9.07 (5), 8.63 (6),
// 9.26 (7); a table of 2^10 or 2^11 entries costs this kernel a resident block per SM.
#define CZ_RANGE_VARIANTS(X)                                                                   \
  X(0, 2, 4, 8, 0, 3) X(1, 2, 4, 8, 0, 4) X(2, 2, 4, 0, 0, 0) X(3, 2, 4, 11, 0, 3) X(4, 2, 4, 8, 0, 0) \
  X(5, 2, 4, 10, 0, 3) X(6, 2, 4, 8, 1, 3) X(7, 2, 4, 11, 0, 4)

cudaError_t launch_range(const RangeArgs& a, int variant, u32 grid, cudaStream_t st) {
  switch (variant) {
#define X(id, rm, mb, win, n64, m)                                                              \
  case id:                                                                                      \
    if (a.negative)                                                                             \
      k_range<rm, mb, false, true><<<grid, RWARPS * 32, RANGE_SMEM, st>>>(a);                   \
    else                                                                                        \
      k_range<rm, mb, false, false, win, n64, m><<<grid, RWARPS * 32, RANGE_SMEM, st>>>(a);    \
    break;
    CZ_RANGE_VARIANTS(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t range_occupancy(int variant, int* bps) {
  switch (variant) {
#define X(id, rm, mb, win, n64, m)                                                                                 \
  case id:                                                                                                         \
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_range<rm, mb, false, false, win, n64, m>,         \
                                                         RWARPS * 32, RANGE_SMEM);
    CZ_RANGE_VARIANTS(X)
#undef X
    default: return cudaErrorInvalidValue;
  }
}

// Opts every range kernel into RANGE_SMEM (> 48 KB) of dynamic shared memory.
cudaError_t range_init() {
  cudaError_t e = cudaSuccess;
#define X(id, rm, mb, win, n64, m)                                                                              \
  if (e == cudaSuccess)                                                                                         \
    e = cudaFuncSetAttribute(k_range<rm, mb, false, false, win, n64, m>,                                       \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RANGE_SMEM);                    \
  if (e == cudaSuccess)                                                                                        \
    e = cudaFuncSetAttribute(k_range<rm, mb, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                             (int)RANGE_SMEM);
  CZ_RANGE_VARIANTS(X)
#undef X
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_range<2, 3, true, false, 8, false, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)RANGE_SMEM);
  return e;
}

cudaError_t launch_range_scout(const RangeArgs& a, const u32* first_seg, u32 nreq, cudaStream_t st) {
  if (!nreq || a.negative) return cudaSuccess;  // the negative variant keeps zero thresholds
  k_range_scout<<<(nreq + 3) / 4, 128, 0, st>>>(a, first_seg, nreq);
  return cudaGetLastError();
}

cudaError_t launch_range_wide(const WidenEntry* list, const u32* count, u32 cap, int limbs, ReqRec* recs,
                              WidenEntry* next, u32 next_cap, u32* next_count, u32 iter_cap, cudaStream_t st,
                              bool negative) {
  const u32 grid = (cap + 127) / 128;
  if (limbs == 6) {
    if (negative)
      k_range_wide<6, true><<<grid, 128, 0, st>>>(list, count, cap, recs, next, next_cap, next_count, iter_cap);
    else
      k_range_wide<6, false><<<grid, 128, 0, st>>>(list, count, cap, recs, next, next_cap, next_count, iter_cap);
  } else {
    if (negative)
      k_range_wide<8, true><<<grid, 128, 0, st>>>(list, count, cap, recs, nullptr, 0, nullptr, iter_cap);
    else
      k_range_wide<8, false><<<grid, 128, 0, st>>>(list, count, cap, recs, nullptr, 0, nullptr, iter_cap);
  }
  return cudaGetLastError();
}

}  // namespace cz
