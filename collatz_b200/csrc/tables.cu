// tables.cu -- device-resident sieve tables, generated on the GPU.
//
//  * Cases mode: the 16 look-ahead bit vectors BV_i and the mod-9 preimage
//    sieve of the reference's precompute() (collatz_cudav7.cu:423-495),
//    bit-identical to it, plus the magic numbers (cu:122-128) and 3^f.
//  * Range mode: the 2^k residue sieve (bit r set iff r mod 2^k cannot be
//    shown to drop within k steps: 3^{f_j(r)} > 2^j for all j <= k) and the
//    survivor table compacted from it, one 16-byte entry per surviving
//    residue with its k-step jump T^k(r) + 1 and exponent f_k(r).
#include <cuda_runtime.h>

#include "common.cuh"
#include "tables.h"

namespace cz {

constexpr u32 NUMERATOR = 306, DENOMINATOR = 485, STEPSIZE = 24;
constexpr u32 ONETHIRD = 2863311531u;

// ------------------------------------------------------------------
// Cases-mode tables.
// ------------------------------------------------------------------

// Dip score of one 24-step parity pattern (cu:431-467).  The reference's
// Odd-Even-Even term (cu:449-453) never fires: its doubleeven() test
// `(x) & 0b11 == 0` (cu:418) parses as `x & (0b11 == 0)`, i.e. 0.
__global__ void k_dipscore(short* __restrict__ maxval) {
  const u32 n0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (n0 >= (1u << STEPSIZE)) return;
  u32 up = 0, n = n0;  // n wraps mod 2^32 exactly like the reference's u32; only parities are used
#pragma unroll
  for (u32 i = 0; i < STEPSIZE; i++) {
    if ((n & 1u) == 0) {
      n = n + n / 2;
      up |= 1u << i;
    } else {
      n = n / 2 + 1;
    }
  }
  int cur = 0, mx = 0;
  u32 evens = 0;
#pragma unroll
  for (u32 i = 0; i < STEPSIZE; i++) {
    if (up & (1u << i)) {
      cur -= (int)(DENOMINATOR - NUMERATOR);
      evens = 0;
    } else {
      cur += (int)NUMERATOR;
      evens += 1;
      if ((evens & 1u) == 0 && cur + (int)(DENOMINATOR - NUMERATOR) > mx) mx = cur + (int)(DENOMINATOR - NUMERATOR);
    }
    if (cur > mx) mx = cur;
  }
  maxval[n0] = (short)mx;
}

// Word w of BV_i: bit p is set iff the residue n0 with (n0 * magic_i) mod
// 2^24 == p has maxval <= cutoff_i (cu:469-479).  n0 = p * 3^f mod 2^24,
// because magic_i = 3^-f mod 2^32.  Words 0..31 are repeated at 2^19.. for
// the funnel shift across the end (cu:475-477).
__global__ void k_bitvectors(const short* __restrict__ maxval, u32* __restrict__ bv, u32 tpo, int firstcutoff) {
  const u32 gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // global word index over 16 vectors
  const u32 lane = lane_id();
  const u32 i = gw >> 19, w = gw & ((1u << 19) - 1);
  if (i >= 16) return;
  u32 p3 = 1;
  for (u32 e = 0; e < tpo + i; e++) p3 *= 3u;
  const u32 p = w * 32 + lane;
  const u32 n0 = (p * p3) & ((1u << STEPSIZE) - 1);
  const int cutoff = firstcutoff + (int)(i * DENOMINATOR);
  const u32 word = __ballot_sync(FULL, (int)maxval[n0] <= cutoff);
  if (lane == 0) {
    bv[(size_t)i * BV_WORDS + w] = word;
    if (w < 32) bv[(size_t)i * BV_WORDS + w + (1u << 19)] = word;
  }
}

// mod9[a][i/32] bit i%32 set iff (a + i * 2^mbi) mod 9 in {0,1,3,6,7} (cu:482-494).
__global__ void k_mod9(u32* __restrict__ mod9, u32 mbi) {
  const u32 t = threadIdx.x;  // 9 * 32 threads, one word each
  if (t >= 9 * 32) return;
  const u32 a = t / 32, wd = t % 32;
  u32 step = 1;
  for (u32 e = 0; e < mbi; e++) step = (step * 2) % 9;
  u32 word = 0;
  for (u32 b = 0; b < 32; b++) {
    const u32 i = wd * 32 + b;
    const u32 red = (a + (i % 9) * step) % 9;
    if (red == 0 || red == 1 || red == 3 || red == 6 || red == 7) word |= 1u << b;
  }
  mod9[t] = word;
}

// magic[i] = ONETHIRD^(tpo+i) mod 2^32 (cu:122-128); pow3[f] = 3^f mod 2^128.
__global__ void k_consts(u32* __restrict__ magic, u32* __restrict__ pow3, u32 tpo) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  u32 m = 1;
  for (u32 i = 1; i < 128; i++) {
    m *= ONETHIRD;
    if (i >= tpo && i - tpo < 16) magic[i - tpo] = m;
  }
  u32 w[4] = {1, 0, 0, 0};
  for (u32 f = 0; f < POW3_COUNT; f++) {
    for (int j = 0; j < 4; j++) pow3[4 * f + j] = w[j];
    u64 c = 0;
    for (int j = 0; j < 4; j++) {
      c += (u64)w[j] * 3u;
      w[j] = (u32)c;
      c >>= 32;
    }
  }
}

// ------------------------------------------------------------------
// Range-mode residue sieve.
// ------------------------------------------------------------------

// 3^f > 2^j, exactly (f <= j <= 64).
__device__ __forceinline__ bool pow3_gt_pow2(u32 f, u32 j, u64 p3) {
  // p3 = 3^f while f <= 40 (3^40 < 2^64); beyond that 3^f > 2^63 >= 2^j for j <= 63
  if (f > 40) return true;
  if (j >= 64) return false;
  return p3 > (1ull << j);
}

// Pass A: the sieve bit array.  One thread per residue, one ballot per word.
__global__ void k_range_bits(u32* __restrict__ bits, u32 k, u64 nres, u32 up) {
  const u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  bool ok = false;
  if (r < nres) {
    u64 n = r, p3 = 1;
    u32 f = 0;
    ok = true;
    for (u32 j = 1; j <= k; j++) {
      if (n & 1) {
        n = n + (n >> 1) + up;  // (3n+1)/2, or (3n-1)/2 for the negative variant (up = 0)
        f++;
        p3 *= 3;
      } else {
        n >>= 1;
      }
      if (!pow3_gt_pow2(f, j, p3)) {
        ok = false;
        break;
      }
    }
  }
  const u32 word = __ballot_sync(FULL, ok);
  if (lane_id() == 0 && r < nres) bits[r >> 5] = word;
}

// Pass B: survivors per chunk of RANGE_CHUNK_WORDS words (vectorised reads).
__global__ void k_range_count(const uint4* __restrict__ bits4, u32* __restrict__ counts, u64 nwords4,
                              u32 nchunks) {
  const u64 c = (u64)blockIdx.x * blockDim.x + threadIdx.x;  // chunk index
  if (c >= nchunks) return;
  const u64 per = RANGE_CHUNK_WORDS / 4;
  u32 cnt = 0;
  for (u64 i = 0; i < per; i++) {
    const u64 idx = c * per + i;
    if (idx < nwords4) {
      const uint4 x = bits4[idx];
      cnt += __popc(x.x) + __popc(x.y) + __popc(x.z) + __popc(x.w);
    }
  }
  counts[c] = cnt;
}

// Exclusive scan of chunk counts in one block (nchunks <= 1024 * 1024).
__global__ void k_scan_counts(const u32* __restrict__ counts, ull* __restrict__ offs, u32 nchunks) {
  __shared__ ull part[1024];
  const u32 t = threadIdx.x;
  const u32 per = (nchunks + 1023) / 1024;
  ull s = 0;
  for (u32 i = 0; i < per; i++) {
    const u32 idx = t * per + i;
    if (idx < nchunks) s += counts[idx];
  }
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    ull acc = 0;
    for (u32 i = 0; i < 1024; i++) {
      const ull x = part[i];
      part[i] = acc;
      acc += x;
    }
    offs[nchunks] = acc;
  }
  __syncthreads();
  ull acc = part[t];
  for (u32 i = 0; i < per; i++) {
    const u32 idx = t * per + i;
    if (idx < nchunks) {
      offs[idx] = acc;
      acc += counts[idx];
    }
  }
}

// Pass C: compact the bit array into the survivor table.  A warp owns one
// chunk; each lane reads one word per step (coalesced), the warp ranks the
// set bits with popc + scan and the owning lanes write entries in residue
// order with their k-step jump.
__global__ void k_range_compact(const u32* __restrict__ bits, const ull* __restrict__ offs,
                                RangeEntry* __restrict__ table, u32 k, u64 nwords, u32 nchunks, u32 up) {
  const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const u32 lane = lane_id();
  if (warp >= nchunks) return;
  ull pos = offs[warp];
  const u64 w0 = (u64)warp * RANGE_CHUNK_WORDS;
  for (u32 s = 0; s < RANGE_CHUNK_WORDS; s += 32) {
    const u64 wi = w0 + s + lane;
    u32 word = (wi < nwords) ? bits[wi] : 0u;
    u32 total;
    const u32 excl = warp_excl_scan(__popc(word), &total);
    ull out = pos + excl;
    while (word) {
      const u32 b = ctz32(word);
      word &= word - 1;
      const u64 r = wi * 32 + b;
      // k-step jump from r (n-space T; parity sequence shared by n == r mod 2^k)
      u64 n = r, p3 = 1;
      u32 f = 0, emax = 0;
      for (u32 j = 1; j <= k; j++) {
        if (n & 1) {
          n = n + (n >> 1) + up;
          f++;
          p3 *= 3;
        } else {
          n >>= 1;
        }
        // e_j = max(0, ceil(log2 3^f) - j): smallest e with 3^f <= 2^(j+e)
        const u32 lg = (f == 0) ? 0u : (64u - __clzll(p3 - 1));
        if (lg > j && lg - j > emax) emax = lg - j;
      }
      RangeEntry e;
      e.r_lo = (u32)r;
      e.meta = (u32)(r >> 32) | (f << 8) | ((u32)(r % 9) << 16) | (emax << 24);
      const u64 c = up ? n + 1 : n - 1;  // T^k(r) + 1, or T'^k(r) - 1 (>= 0: survivors have r >= 1)
      e.c_lo = (u32)c;
      e.c_hi = (u32)(c >> 32);
      table[out++] = e;
    }
    pos += total;
  }
}

// For every removed residue r: with tau the first j where 3^{f_j} < 2^j,
// T^tau(2^k + r) < 2^k + r must hold.  Since T^tau is affine with slope
// 3^f / 2^tau < 1 on the class, this proves the sieve for all n >= 2^k.
__global__ void k_range_validate(const u32* __restrict__ bits, u32 k, u64 nres, ull* __restrict__ bad, u32 up) {
  const u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nres) return;
  if ((bits[r >> 5] >> (r & 31)) & 1u) return;
  u64 n = r, p3 = 1;
  u32 f = 0, tau = 0;
  for (u32 j = 1; j <= k; j++) {
    if (n & 1) {
      n = n + (n >> 1) + up;
      f++;
      p3 *= 3;
    } else {
      n >>= 1;
    }
    if (!pow3_gt_pow2(f, j, p3)) {
      tau = j;
      break;
    }
  }
  // x = 2^k + r in two limbs (k <= 40 keeps x < 2^41; values stay < 2^64 for tau <= k)
  const u64 s = (1ull << k) + r;
  u64 x = s;
  for (u32 j = 0; j < tau; j++) x = (x & 1) ? x + (x >> 1) + up : x >> 1;
  if (tau == 0 || !(x < s)) atomicAdd(bad, 1ull);
}

// ------------------------------------------------------------------
// Host entry points (called by the runtime in api.cu).
// ------------------------------------------------------------------

cudaError_t build_case_tables(CaseTables* t, u32 maxbits, cudaStream_t st) {
  t->maxbits = maxbits;
  t->mbi = maxbits - 10;
  t->tpo = t->mbi * NUMERATOR / DENOMINATOR + 1;
  cudaError_t e;
  if ((e = cudaMalloc(&t->bv, sizeof(u32) * 16 * BV_WORDS))) return e;
  if ((e = cudaMalloc(&t->mod9, sizeof(u32) * 9 * 32))) return e;
  if ((e = cudaMalloc(&t->magic, sizeof(u32) * 16))) return e;
  if ((e = cudaMalloc(&t->pow3, sizeof(u32) * 4 * POW3_COUNT))) return e;
  short* maxval = nullptr;
  if ((e = cudaMalloc(&maxval, sizeof(short) << STEPSIZE))) return e;
  k_dipscore<<<(1u << STEPSIZE) / 256, 256, 0, st>>>(maxval);
  const int firstcutoff = (short)(DENOMINATOR * t->tpo - NUMERATOR * t->mbi);  // cu:424
  k_bitvectors<<<(16u << 19) * 32 / 256, 256, 0, st>>>(maxval, t->bv, t->tpo, firstcutoff);
  k_mod9<<<1, 9 * 32, 0, st>>>(t->mod9, t->mbi);
  k_consts<<<1, 32, 0, st>>>(t->magic, t->pow3, t->tpo);
  if ((e = cudaGetLastError())) return e;
  if ((e = cudaStreamSynchronize(st))) return e;
  cudaFree(maxval);
  return cudaSuccess;
}

void free_case_tables(CaseTables* t) {
  cudaFree(t->bv);
  cudaFree(t->mod9);
  cudaFree(t->magic);
  cudaFree(t->pow3);
  t->bv = t->mod9 = t->magic = t->pow3 = nullptr;
}

// Pass D: stable partition of the residue-ordered table by r mod 9 into
// class-major order.  One warp per block of CLS_BLOCK entries: D1 counts
// each class (hist[c * nblk + block]), an exclusive scan of hist in that
// order gives every (class, block) its output offset, and D2 scatters the
// block's entries with one ballot per class per 32 entries, which keeps
// residue order inside each class.
constexpr u32 CLS_BLOCK = 2048;

__global__ void k_class_hist(const RangeEntry* __restrict__ t, u64 n, u32* __restrict__ hist, u32 nblk) {
  const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = lane_id();
  if (warp >= nblk) return;
  u32 cnt[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (u32 i = lane; i < CLS_BLOCK; i += 32) {
    const u64 idx = (u64)warp * CLS_BLOCK + i;
    if (idx < n) {
      const u32 c = (t[idx].meta >> 16) & 0xFFu;
#pragma unroll
      for (u32 j = 0; j < 9; j++) cnt[j] += (c == j);
    }
  }
#pragma unroll
  for (u32 j = 0; j < 9; j++) {
    u32 x = cnt[j];
#pragma unroll
    for (u32 d = 16; d; d >>= 1) x += __shfl_xor_sync(FULL, x, d);
    if (lane == 0) hist[j * nblk + warp] = x;
  }
}

__global__ void k_class_scatter(const RangeEntry* __restrict__ t, u64 n, const ull* __restrict__ offs, u32 nblk,
                                RangeEntry* __restrict__ out) {
  const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = lane_id();
  if (warp >= nblk) return;
  ull base[9];
#pragma unroll
  for (u32 j = 0; j < 9; j++) base[j] = offs[j * nblk + warp];
  const u32 lt = lanemask_lt();
  for (u32 i = 0; i < CLS_BLOCK; i += 32) {
    const u64 idx = (u64)warp * CLS_BLOCK + i + lane;
    const bool ok = idx < n;
    RangeEntry e{0, 0, 0, 0};
    if (ok) e = t[idx];
    const u32 c = ok ? ((e.meta >> 16) & 0xFFu) : 9u;
    ull pos = 0;
#pragma unroll
    for (u32 j = 0; j < 9; j++) {
      const u32 m = __ballot_sync(FULL, c == j);
      if (c == j) pos = base[j] + __popc(m & lt);
      base[j] += __popc(m);
    }
    if (ok) out[pos] = e;
  }
}

cudaError_t build_range_table(RangeTable* t, u32 k, bool validate, cudaStream_t st, bool negative) {
  t->k = k;
  const u64 nres = 1ull << k;
  const u64 nwords = (nres + 31) / 32;
  const u64 nwords_pad = ((nwords + RANGE_CHUNK_WORDS - 1) / RANGE_CHUNK_WORDS) * RANGE_CHUNK_WORDS;
  const u32 nchunks = (u32)(nwords_pad / RANGE_CHUNK_WORDS);
  cudaError_t e;
  if ((e = cudaMalloc(&t->bits, nwords_pad * 4))) return e;
  if ((e = cudaMemsetAsync(t->bits, 0, nwords_pad * 4, st))) return e;
  u32* counts = nullptr;
  ull* offs = nullptr;
  if ((e = cudaMalloc(&counts, sizeof(u32) * nchunks))) return e;
  if ((e = cudaMalloc(&offs, sizeof(ull) * (nchunks + 1)))) return e;
  const u32 tpb = 256;
  const u32 up = negative ? 0u : 1u;
  t->negative = negative;
  k_range_bits<<<(u32)((nres + tpb - 1) / tpb), tpb, 0, st>>>(t->bits, k, nres, up);
  k_range_count<<<(nchunks + 127) / 128, 128, 0, st>>>((const uint4*)t->bits, counts, nwords_pad / 4, nchunks);
  k_scan_counts<<<1, 1024, 0, st>>>(counts, offs, nchunks);
  ull total = 0;
  if ((e = cudaMemcpyAsync(&total, offs + nchunks, sizeof(ull), cudaMemcpyDeviceToHost, st))) return e;
  if ((e = cudaStreamSynchronize(st))) return e;
  t->count = total;
  if ((e = cudaMalloc(&t->table, sizeof(RangeEntry) * (total ? total : 1)))) return e;
  k_range_compact<<<(nchunks * 32 + 255) / 256, 256, 0, st>>>(t->bits, offs, t->table, k, nwords, nchunks, up);
  t->violations = 0;
  if (validate) {
    ull* bad = nullptr;
    if ((e = cudaMalloc(&bad, sizeof(ull)))) return e;
    cudaMemsetAsync(bad, 0, sizeof(ull), st);
    k_range_validate<<<(u32)((nres + tpb - 1) / tpb), tpb, 0, st>>>(t->bits, k, nres, bad, up);
    cudaMemcpyAsync(&t->violations, bad, sizeof(ull), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    cudaFree(bad);
  }
  if ((e = cudaGetLastError())) return e;
  if ((e = cudaStreamSynchronize(st))) return e;
  cudaFree(counts);
  cudaFree(offs);
  // class-major order (pass D)
  const u32 nblk = (u32)((total + CLS_BLOCK - 1) / CLS_BLOCK);
  for (int c = 0; c < 10; c++) t->cls[c] = 0;
  if (nblk) {
    u32* hist = nullptr;
    ull* coffs = nullptr;
    RangeEntry* out = nullptr;
    if ((e = cudaMalloc(&hist, sizeof(u32) * 9 * nblk))) return e;
    if ((e = cudaMalloc(&coffs, sizeof(ull) * (9 * nblk + 1)))) return e;
    if ((e = cudaMalloc(&out, sizeof(RangeEntry) * total))) return e;
    const u32 wpb = 8;  // warps per block
    k_class_hist<<<(nblk + wpb - 1) / wpb, 32 * wpb, 0, st>>>(t->table, total, hist, nblk);
    k_scan_counts<<<1, 1024, 0, st>>>(hist, coffs, 9 * nblk);
    k_class_scatter<<<(nblk + wpb - 1) / wpb, 32 * wpb, 0, st>>>(t->table, total, coffs, nblk, out);
    for (int c = 0; c < 9 && !e; c++)
      e = cudaMemcpyAsync(&t->cls[c], coffs + (size_t)c * nblk, sizeof(ull), cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaGetLastError();
    if (!e) e = cudaStreamSynchronize(st);
    cudaFree(hist);
    cudaFree(coffs);
    cudaFree(t->table);
    t->table = out;
    if (e) return e;
  }
  t->cls[9] = total;
  return cudaSuccess;
}

void free_range_table(RangeTable* t) {
  cudaFree(t->bits);
  cudaFree(t->table);
  t->bits = nullptr;
  t->table = nullptr;
}

}  // namespace cz
