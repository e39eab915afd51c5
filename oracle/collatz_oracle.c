/*
 * collatz_oracle.c -- CPU oracle for the collatz_b200 hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see collatz_oracle.h).  Plain C11 with
 * unsigned __int128; deliberately simple and scalar so that it can be
 * read against the reference line by line.
 */
#include "collatz_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef orc_u128 u128;

/* Reference constants (collatz_cudav7.cu:43-55). */
#define NUMERATOR 306u
#define DENOMINATOR 485u
#define LASTBITS 10u
#define STEPSIZE 24u
#define BATCHSIZE (1u << 16)
#define ONETHIRD 2863311531u
#define CUTOFFPOWER 100u

/* THREEPOWERSU32, cu:57-59. */
static const uint32_t P3[17] = {1,       3,       9,        27,      81,
                                243,     729,     2187,     6561,    19683,
                                59049,   177147,  531441,   1594323, 4782969,
                                14348907, 43046721};

static u128 pow3(unsigned e) {
  u128 x = 1;
  while (e--) x *= 3;
  return x;
}

static unsigned ctz32(uint32_t x) { return (unsigned)__builtin_ctz(x); }

#define U128_OF(lo, hi) (((u128)(hi) << 64) | (u128)(lo))

/* ===================================================================== */
/* Tables: magic numbers (cu:122-128), bit vectors + mod-9 sieve          */
/* (precompute, cu:423-495).                                              */
/* ===================================================================== */

int orc_tables_init(orc_tables *t, uint32_t maxbits) {
  if (maxbits < 16 || maxbits > 96) return -1;
  memset(t, 0, sizeof *t);
  t->maxbits = maxbits;
  t->mbi = maxbits - LASTBITS;
  t->tpo = t->mbi * NUMERATOR / DENOMINATOR + 1;

  /* magicnumbers[i - TPO] = ONETHIRD^i mod 2^32 (cu:122-128) */
  uint32_t m = 1;
  for (uint32_t i = 1; i < 128; i++) {
    m *= ONETHIRD;
    if (i >= t->tpo && i - t->tpo < 16) t->magic[i - t->tpo] = m;
  }

  t->bv = (uint32_t *)calloc((size_t)16 * ORC_BV_WORDS, sizeof(uint32_t));
  if (!t->bv) return -2;

  /* cu:424-426: the first cutoff goes through an i16 cast. */
  int32_t firstcutoff = (int16_t)(DENOMINATOR * t->tpo - NUMERATOR * t->mbi);
  int32_t cutoffs[16];
  for (int i = 0; i < 16; i++) cutoffs[i] = firstcutoff + i * (int32_t)DENOMINATOR;

  for (uint32_t n0 = 0; n0 < (1u << STEPSIZE); n0++) {
    /* parity word in the "+1" space (cu:431-441): bit i = odd step */
    uint32_t upordown = 0;
    uint64_t n = n0;
    for (unsigned i = 0; i < STEPSIZE; i++) {
      if (n % 2 == 0) {
        n = n + n / 2;
        upordown |= 1u << i;
      } else {
        n = n / 2 + 1;
      }
    }
    /* dip score (cu:442-467).  The Odd-Even-Even term of cu:449-453 calls
     * doubleeven(), whose test `(x) & 0b11 == 0` (cu:418) parses as
     * `x & (0b11 == 0)` == 0, so it never fires; it is omitted here. */
    int32_t curval = 0, maxval = 0;
    uint32_t numevens = 0;
    for (unsigned i = 0; i < STEPSIZE; i++) {
      if (upordown & (1u << i)) {
        curval -= (int32_t)(DENOMINATOR - NUMERATOR);
        numevens = 0;
      } else {
        curval += (int32_t)NUMERATOR;
        numevens += 1;
        if (numevens % 2 == 0) { /* Path-Merging term, cu:459-464 */
          if (curval + (int32_t)(DENOMINATOR - NUMERATOR) > maxval)
            maxval = curval + (int32_t)(DENOMINATOR - NUMERATOR);
        }
      }
      if (curval > maxval) maxval = curval;
    }
    /* cu:469-479 */
    for (int a = 0; a < 16; a++) {
      if (maxval <= cutoffs[a]) {
        uint32_t index = (n0 * t->magic[a]) & ((1u << STEPSIZE) - 1);
        uint32_t *bv = t->bv + (size_t)a * ORC_BV_WORDS;
        bv[index / 32] |= 1u << (index % 32);
        if (index / 32 < 32) bv[index / 32 + (1u << 19)] |= 1u << (index % 32);
      }
    }
  }

  /* Mod 9 preimage sieve, cu:482-494: bit i of row a is set iff
   * (a + i * 2^(N-A)) mod 9 is in {0,1,3,6,7}. */
  uint32_t step = (uint32_t)(((u128)1 << t->mbi) % 9);
  for (uint32_t a = 0; a < 9; a++) {
    uint32_t red = a;
    for (uint32_t i = 0; i < (1u << LASTBITS); i++) {
      if (red == 0 || red == 1 || red == 3 || red == 6 || red == 7)
        t->mod9[a][i / 32] |= 1u << (i % 32);
      red += step;
      if (red >= 9) red -= 9;
    }
  }
  return 0;
}

void orc_tables_free(orc_tables *t) {
  free(t->bv);
  t->bv = NULL;
}

void orc_case_result_init(orc_case_result *r) {
  uint64_t *buf = r->overflow;
  uint64_t cap = r->overflow_cap;
  memset(r, 0, sizeof *r);
  r->overflow = buf;
  r->overflow_cap = cap;
}

/* ===================================================================== */
/* Step 2 + Step 3 for one pair (compute_kernel cu:185-411 and            */
/* search2/search3 cu:654-715).                                           */
/* ===================================================================== */

static void note_overflow(orc_case_result *r, u128 seed) {
  if (r->overflow && r->n_overflow < r->overflow_cap) {
    r->overflow[2 * r->n_overflow] = (uint64_t)seed;
    r->overflow[2 * r->n_overflow + 1] = (uint64_t)(seed >> 64);
  }
  r->n_overflow++;
}

/* Iterates one seed with the reference's checkpoint structure:
 * [odd run (<= 8), overflow test, even run (<= 31)] x 2, hash ^= low limb,
 * stop when v < n (cu:280-405; search3 cu:684-715).  v = T^k(n) + 1.
 * Also tracks sigma and E as defined in collatz_oracle.h. */
static uint32_t seed_cases(u128 n, u128 v, uint32_t mbi, int cpu_sem,
                           orc_case_result *r) {
  const u128 CUT = (u128)1 << CUTOFFPOWER;
  uint32_t hash = 0;
  int found = 0, ovf = 0;
  uint64_t st = mbi;
  u128 E = v - 1;
  if (n < 3) return 0; /* v < n is unreachable: the reference loops forever */
  for (;;) {
    r->checkpoints++;
    for (int half = 0; half < 2; half++) {
      unsigned a = ctz32((uint32_t)v | (1u << 8));
      v = (v >> a) * P3[a];
      if (!found) st += a;
      /* GPU: both tests are >= (cu:295, 334); CPU search3: >= then >
       * (cu:690, 702). */
      int o = (half == 1 && cpu_sem) ? (v > CUT) : (v >= CUT);
      if (o) {
        note_overflow(r, n);
        ovf = 1;
        v = 2;
      } else if (!found && !ovf && v - 1 > E) {
        E = v - 1;
      }
      u128 m = v - 1;
      unsigned b = ctz32((uint32_t)m | 0x80000000u);
      if (!found && !ovf) {
        if ((m >> b) < n) {
          unsigned i = 1;
          while ((m >> i) >= n) i++;
          st += i;
          found = 1;
        } else {
          st += b;
        }
      }
      v = (m >> b) + 1;
    }
    hash ^= (uint32_t)v;
    if (v < n) break;
  }
  if (!ovf) {
    u128 me = U128_OF(r->max_exc[0], r->max_exc[1]);
    u128 mes = U128_OF(r->max_exc_seed[0], r->max_exc_seed[1]);
    u128 mss = U128_OF(r->max_st_seed[0], r->max_st_seed[1]);
    int first = r->seeds_done++ == 0;
    if (first || E > me || (E == me && n < mes)) {
      r->max_exc[0] = (uint64_t)E;
      r->max_exc[1] = (uint64_t)(E >> 64);
      r->max_exc_seed[0] = (uint64_t)n;
      r->max_exc_seed[1] = (uint64_t)(n >> 64);
    }
    if (first || st > r->max_st || (st == r->max_st && n < mss)) {
      r->max_st = st;
      r->max_st_seed[0] = (uint64_t)n;
      r->max_st_seed[1] = (uint64_t)(n >> 64);
    }
  }
  return hash;
}

static uint32_t pair_impl(const orc_tables *t, uint32_t bigindex, u128 base,
                          u128 number, int cpu_sem, orc_case_result *r) {
  uint32_t hash = 0;
  uint32_t f = t->tpo + bigindex;
  u128 tp = pow3(f);
  uint32_t redmod9 = (uint32_t)(base % 9);
  for (uint32_t a = 0; a < 32; a++) {
    uint32_t w = t->mod9[redmod9][a];
    if (bigindex < 16) {
      uint32_t index = (t->magic[bigindex] * (uint32_t)number) & ((1u << STEPSIZE) - 1);
      const uint32_t *bv = t->bv + (size_t)bigindex * ORC_BV_WORDS;
      uint64_t both = ((uint64_t)bv[index / 32 + a + 1] << 32) | bv[index / 32 + a];
      w &= (uint32_t)(both >> (index % 32));
    }
    while (w) {
      uint32_t hi = 32 * a + ctz32(w);
      w &= w - 1;
      u128 n = base + ((u128)hi << t->mbi);
      u128 v = number + (u128)hi * tp;
      r->seeds++;
      hash ^= seed_cases(n, v, t->mbi, cpu_sem, r);
    }
  }
  return hash;
}

uint32_t orc_pair(const orc_tables *t, uint32_t bigindex, uint64_t base_lo,
                  uint64_t base_hi, uint64_t number_lo, uint64_t number_hi,
                  int cpu_sem, orc_case_result *r) {
  return pair_impl(t, bigindex, U128_OF(base_lo, base_hi),
                   U128_OF(number_lo, number_hi), cpu_sem, r);
}

/* ===================================================================== */
/* Step 1 (search1, cu:497-563).                                          */
/* ===================================================================== */

typedef struct {
  const orc_tables *t;
  orc_leaf_cb leaf;
  orc_root_cb root;
  void *ctx;
  uint32_t cut;
  u128 p3[96];
} s1_state;

static void search1_rec(s1_state *s, u128 base, uint32_t sigfig, uint32_t tp,
                        u128 number, uint32_t de, uint32_t ne) {
  const uint32_t mbi = s->t->mbi;
  /* Induction sieve, cu:507 (u32 arithmetic as in the reference). */
  if (DENOMINATOR * tp <= NUMERATOR * sigfig) return;
  /* Mod 3 preimage sieve, cu:509-511. */
  if (ne >= 2 && ne % 2 == 0) {
    if (NUMERATOR * (sigfig - 1) >= DENOMINATOR * (tp - 1)) return;
  }
  if (s->root && sigfig == s->cut) {
    s->root(s->ctx, (uint64_t)base, (uint64_t)(base >> 64), sigfig, tp,
            (uint64_t)number, (uint64_t)(number >> 64), de, ne);
    return;
  }
  if (sigfig == mbi) {
    if (s->leaf)
      s->leaf(s->ctx, tp - s->t->tpo, (uint64_t)base, (uint64_t)(base >> 64),
              (uint64_t)number, (uint64_t)(number >> 64));
    return;
  }
  uint32_t doubleinplay = (NUMERATOR * (sigfig + 1) >= DENOMINATOR * tp) ? 1u : 0u;
  u128 numberA = number;
  u128 numberB = number + s->p3[tp];
  if (number % 2 == 0) {
    search1_rec(s, base, sigfig + 1, tp + 1, numberA + numberA / 2,
                (de | doubleinplay) & ~2u, 0);
    if (de < 2)
      search1_rec(s, base | ((u128)1 << sigfig), sigfig + 1, tp, numberB / 2 + 1,
                  de << 1, ne + 1);
  } else {
    if (de < 2)
      search1_rec(s, base, sigfig + 1, tp, numberA / 2 + 1, de << 1, ne + 1);
    search1_rec(s, base | ((u128)1 << sigfig), sigfig + 1, tp + 1,
                numberB + numberB / 2, (de | doubleinplay) & ~2u, 0);
  }
}

static void s1_init(s1_state *s, const orc_tables *t) {
  memset(s, 0, sizeof *s);
  s->t = t;
  u128 a = 1;
  for (int i = 0; i < 96; i++) {
    s->p3[i] = a;
    a *= 3;
  }
}

int orc_search1(const orc_tables *t, uint64_t base_lo, uint64_t base_hi,
                uint32_t sigfig, uint32_t tp, uint64_t number_lo,
                uint64_t number_hi, uint32_t de, uint32_t ne, orc_leaf_cb cb,
                void *ctx) {
  u128 base = U128_OF(base_lo, base_hi), number = U128_OF(number_lo, number_hi);
  if (sigfig > t->mbi) return -1;
  s1_state s;
  s1_init(&s, t);
  s.leaf = cb;
  s.ctx = ctx;
  search1_rec(&s, base, sigfig, tp, number, de, ne);
  return 0;
}

int orc_split(const orc_tables *t, uint64_t base_lo, uint64_t base_hi,
              uint32_t sigfig, uint32_t tp, uint64_t number_lo,
              uint64_t number_hi, uint32_t de, uint32_t ne, uint32_t cut,
              orc_root_cb cb, void *ctx) {
  u128 base = U128_OF(base_lo, base_hi), number = U128_OF(number_lo, number_hi);
  if (sigfig > t->mbi || cut >= t->mbi || cut < sigfig) return -1;
  s1_state s;
  s1_init(&s, t);
  s.root = cb;
  s.ctx = ctx;
  s.cut = cut;
  search1_rec(&s, base, sigfig, tp, number, de, ne);
  return 0;
}

typedef struct {
  const orc_tables *t;
  orc_case_result *r;
  uint64_t count[16];
} run_state;

static void run_leaf(void *ctx, uint32_t bigindex, uint64_t blo, uint64_t bhi,
                     uint64_t nlo, uint64_t nhi) {
  run_state *rs = (run_state *)ctx;
  u128 base = U128_OF(blo, bhi), number = U128_OF(nlo, nhi);
  if (bigindex >= 16) { /* CPU fallback, cu:517-519 */
    rs->r->cpu_pairs++;
    rs->r->hash ^= pair_impl(rs->t, bigindex, base, number, 1, rs->r);
    return;
  }
  rs->count[bigindex]++;
  rs->r->pairs++;
  rs->r->hash ^= pair_impl(rs->t, bigindex, base, number, 0, rs->r);
}

int orc_run_case(const orc_tables *t, uint64_t base_lo, uint64_t base_hi,
                 uint32_t sigfig, uint32_t tp, uint64_t number_lo,
                 uint64_t number_hi, uint32_t de, uint32_t ne,
                 orc_case_result *r) {
  run_state rs;
  memset(&rs, 0, sizeof rs);
  rs.t = t;
  rs.r = r;
  int rc = orc_search1(t, base_lo, base_hi, sigfig, tp, number_lo, number_hi,
                       de, ne, run_leaf, &rs);
  if (rc) return rc;
  /* one launch per full bucket (cu:532-534) plus one per non-empty bucket
   * at the final flush (cu:177-179) */
  for (int b = 0; b < 16; b++) r->launches += (rs.count[b] + BATCHSIZE - 1) / BATCHSIZE;
  return 0;
}

/* ===================================================================== */
/* Range mode.                                                           */
/* ===================================================================== */

/* 1 iff residue r mod 2^k survives the k-step descent sieve:
 * 3^{f_j(r)} >= 2^j for every 1 <= j <= k (f_j = odd steps among the first j). */
static int residue_survives_v(uint64_t r, uint32_t k, int neg) {
  uint64_t n = r;
  unsigned f = 0;
  for (unsigned j = 1; j <= k; j++) {
    if (n & 1) {
      n = n + (n >> 1) + (neg ? 0 : 1);  /* (3n+1)/2, or (3n-1)/2 for T' */
      f++;
    } else {
      n >>= 1;
    }
    if (pow3(f) < ((u128)1 << j)) return 0;
  }
  return 1;
}
static int residue_survives(uint64_t r, uint32_t k) { return residue_survives_v(r, k, 0); }

uint64_t orc_range_sieve(uint32_t k, uint8_t *bits) {
  uint64_t count = 0;
  uint64_t nres = 1ull << k;
  if (bits) memset(bits, 0, (size_t)(nres + 7) / 8);
  for (uint64_t r = 0; r < nres; r++) {
    if (residue_survives(r, k)) {
      count++;
      if (bits) bits[r >> 3] |= (uint8_t)(1u << (r & 7));
    }
  }
  return count;
}

/* Sieve tables kept for the life of the process, one per k <= 26, built on
 * first use under a lock (repeated range calls then pay for the table once). */
static pthread_mutex_t g_sieve_mu = PTHREAD_MUTEX_INITIALIZER;
static uint8_t *g_sieve[27];
static const uint8_t *cached_sieve(uint32_t k) {
  if (k == 0 || k > 26) return NULL;
  pthread_mutex_lock(&g_sieve_mu);
  if (!g_sieve[k]) {
    uint8_t *b = (uint8_t *)malloc((size_t)((1ull << k) + 7) / 8);
    if (b) orc_range_sieve(k, b);
    g_sieve[k] = b;
  }
  const uint8_t *out = g_sieve[k];
  pthread_mutex_unlock(&g_sieve_mu);
  return out;
}
/* The first j <= k0 parity steps of r depend only on r mod 2^k0, so a residue
 * removed by the 2^k0 sieve is removed by every 2^k sieve with k >= k0: the
 * direct test of a large k first looks r mod 2^20 up in the cached table. */
#define DIRECT_PREFILTER_K 20u

uint64_t orc_range_sieve_validate(uint32_t k) {
  uint64_t bad = 0;
  for (uint64_t r = 0; r < (1ull << k); r++) {
    uint64_t n = r;
    unsigned f = 0, tau = 0;
    for (unsigned j = 1; j <= k; j++) {
      if (n & 1) {
        n = n + (n >> 1) + 1;
        f++;
      } else {
        n >>= 1;
      }
      if (pow3(f) < ((u128)1 << j)) {
        tau = j;
        break;
      }
    }
    if (!tau) continue;
    u128 s = ((u128)1 << k) + r, x = s;
    for (unsigned j = 0; j < tau; j++) x = (x & 1) ? x + (x >> 1) + 1 : x >> 1;
    if (!(x < s)) bad++;
  }
  return bad;
}

/* 512-bit unsigned values as 8 x u64, little-endian, for the rare seeds
 * that leave 128 bits and for trajectory queries. */
typedef struct {
  uint64_t w[8];
} big;

static void big_from_u32(big *x, const uint32_t *limbs, unsigned nl) {
  memset(x, 0, sizeof *x);
  for (unsigned i = 0; i < nl && i < 16; i++) x->w[i / 2] |= (uint64_t)limbs[i] << (32 * (i % 2));
}
static void big_to_u32(const big *x, uint32_t *limbs) {
  for (int i = 0; i < 16; i++) limbs[i] = (uint32_t)(x->w[i / 2] >> (32 * (i % 2)));
}
static int big_cmp(const big *a, const big *b) {
  for (int i = 7; i >= 0; i--) {
    if (a->w[i] != b->w[i]) return a->w[i] < b->w[i] ? -1 : 1;
  }
  return 0;
}
static void big_shr1(big *x) {
  for (int i = 0; i < 7; i++) x->w[i] = (x->w[i] >> 1) | (x->w[i + 1] << 63);
  x->w[7] >>= 1;
}
/* x <- (3x+1)/2 = x + (x>>1) + 1 for odd x (cin = 1), or the negative
 * variant's (3x-1)/2 = x + (x>>1) (cin = 0); returns 1 on overflow */
static int big_odd_step_c(big *x, unsigned cin) {
  big h = *x;
  big_shr1(&h);
  unsigned __int128 c = cin;
  for (int i = 0; i < 8; i++) {
    c += (unsigned __int128)x->w[i] + h.w[i];
    x->w[i] = (uint64_t)c;
    c >>= 64;
  }
  return c != 0;
}

/* Steps after which a seed of the negative variant counts as not
 * descending (the known non-descending seeds, the cycle minima 5 and 17,
 * are caught exactly by returning to themselves). */
#define NEG_STEP_CAP (1u << 22)

/* sigma and E of one seed with single steps on 512-bit values (T, or T'
 * when neg).  Returns 0 ok, 2 overflow, 3 (neg) returned to the seed or
 * reached the step cap: the seed does not descend. */
static int big_seed_v(const big *n, uint64_t *st_out, big *E_out, uint64_t *steps, int neg) {
  big x = *n, E = *n;
  uint64_t st = 0;
  for (;;) {
    if (x.w[0] & 1) {
      if (big_odd_step_c(&x, neg ? 0u : 1u)) return 2;
      if (big_cmp(&x, &E) > 0) E = x;
    } else {
      big_shr1(&x);
    }
    st++;
    if (big_cmp(&x, n) < 0) break;
    if (neg && (big_cmp(&x, n) == 0 || st >= NEG_STEP_CAP)) return 3;
  }
  *st_out = st;
  *E_out = E;
  if (steps) *steps += st;
  return 0;
}
static int big_seed(const big *n, uint64_t *st_out, big *E_out, uint64_t *steps) {
  return big_seed_v(n, st_out, E_out, steps, 0);
}

typedef struct {
  uint64_t seeds, failures, steps, odd_runs, even_runs, wide64;
  big E;
  u128 E_seed;
  uint64_t st;
  u128 st_seed;
  int have;
} range_acc;

static void acc_seed(range_acc *a, u128 n, uint64_t st, const big *E) {
  if (!a->have) {
    a->have = 1;
    a->E = *E;
    a->E_seed = n;
    a->st = st;
    a->st_seed = n;
    return;
  }
  int c = big_cmp(E, &a->E);
  if (c > 0 || (c == 0 && n < a->E_seed)) {
    a->E = *E;
    a->E_seed = n;
  }
  if (st > a->st || (st == a->st && n < a->st_seed)) {
    a->st = st;
    a->st_seed = n;
  }
}

static void acc_merge(range_acc *a, const range_acc *b) {
  a->seeds += b->seeds;
  a->failures += b->failures;
  a->steps += b->steps;
  a->odd_runs += b->odd_runs;
  a->even_runs += b->even_runs;
  a->wide64 += b->wide64;
  if (!b->have) return;
  if (!a->have) {
    a->have = 1;
    a->E = b->E;
    a->E_seed = b->E_seed;
    a->st = b->st;
    a->st_seed = b->st_seed;
    return;
  }
  int c = big_cmp(&b->E, &a->E);
  if (c > 0 || (c == 0 && b->E_seed < a->E_seed)) {
    a->E = b->E;
    a->E_seed = b->E_seed;
  }
  if (b->st > a->st || (b->st == a->st && b->st_seed < a->st_seed)) {
    a->st = b->st;
    a->st_seed = b->st_seed;
  }
}

static void big_from_u128(big *x, u128 v) {
  memset(x, 0, sizeof *x);
  x->w[0] = (uint64_t)v;
  x->w[1] = (uint64_t)(v >> 64);
}

static const u128 U128_MAX = ~(u128)0;

/* method 0: single T-steps in u128; 512-bit path on overflow. */
static void seed_steps(range_acc *a, u128 n) {
  u128 x = n, E = n;
  uint64_t st = 0;
  for (;;) {
    if (x & 1) {
      if (x > (U128_MAX - 1) / 3) goto wide;
      x = x + (x >> 1) + 1;
      if (x > E) E = x;
    } else {
      x >>= 1;
    }
    st++;
    if (x < n) break;
  }
  {
    big Eb;
    big_from_u128(&Eb, E);
    a->steps += st;
    acc_seed(a, n, st, &Eb);
    return;
  }
wide : {
  big nb, Eb;
  big_from_u128(&nb, n);
  uint64_t st2;
  if (big_seed(&nb, &st2, &Eb, &a->steps)) {
    a->failures++;
    return;
  }
  acc_seed(a, n, st2, &Eb);
}
}

/* method 1: the reference's run-length loop (search3, cu:684-715) in the
 * "+1" space, v = T^k(n) + 1: odd run a = ctz(v | 2^8), v = 3^a (v >> a);
 * even run b = ctz((v-1) | 2^31), v = ((v-1) >> b) + 1.  Descent can only
 * happen inside an even run, so the exact step is recovered there. */
static void seed_runs(range_acc *a, u128 n) {
  u128 v = n + 1, E = n;
  uint64_t st = 0;
  for (;;) {
    unsigned oa = ctz32((uint32_t)v | (1u << 8));
    u128 q = v >> oa;
    if (q > U128_MAX / P3[oa]) goto wide;
    v = q * P3[oa];
    st += oa;
    a->odd_runs++;
    if (v - 1 > E) E = v - 1;
    u128 m = v - 1;
    unsigned b = ctz32((uint32_t)m | 0x80000000u);
    a->even_runs++;
    if ((m >> b) < n) {
      unsigned i = 1;
      while ((m >> i) >= n) i++;
      st += i;
      break;
    }
    st += b;
    v = (m >> b) + 1;
  }
  {
    big Eb;
    big_from_u128(&Eb, E);
    a->steps += st;
    acc_seed(a, n, st, &Eb);
    return;
  }
wide : {
  big nb, Eb;
  big_from_u128(&nb, n);
  uint64_t st2;
  if (big_seed(&nb, &st2, &Eb, &a->steps)) {
    a->failures++;
    return;
  }
  acc_seed(a, n, st2, &Eb);
}
}

/* method 3: method 1 in uint64_t with overflow detection.  The odd run's
 * multiply 3^a (v >> a) is checked with __builtin_mul_overflow; the even
 * run only shrinks the value.  A seed whose value would leave 64 bits is
 * re-run with the 128-bit method 1 (counted in wide64), so the results
 * equal method 1's. */
static void seed_runs64(range_acc *a, u128 n128) {
  if (n128 >> 63) {
    a->wide64++;
    seed_runs(a, n128);
    return;
  }
  const uint64_t n = (uint64_t)n128;
  uint64_t v = n + 1, E = n, st = 0;
  uint64_t odd = 0, even = 0;
  for (;;) {
    unsigned oa = ctz32((uint32_t)v | (1u << 8));
    uint64_t w;
    if (__builtin_mul_overflow(v >> oa, (uint64_t)P3[oa], &w)) {
      a->wide64++;
      seed_runs(a, n128);
      return;
    }
    v = w;
    st += oa;
    odd++;
    if (v - 1 > E) E = v - 1;
    const uint64_t m = v - 1;
    unsigned b = ctz32((uint32_t)m | 0x80000000u);
    even++;
    if ((m >> b) < n) {
      unsigned i = 1;
      while ((m >> i) >= n) i++;
      st += i;
      break;
    }
    st += b;
    v = (m >> b) + 1;
  }
  big Eb;
  big_from_u128(&Eb, E);
  a->steps += st;
  a->odd_runs += odd;
  a->even_runs += even;
  acc_seed(a, n128, st, &Eb);
}

/* method 2: the device kernel's structure for sieved seeds n >= 2^k: the
 * first k steps as one jump (no descent is possible there for a survivor),
 * then the run-length loop of method 1.  Counts only the runs after the
 * jump (the work model of the GPU kernel). */
static void seed_jump_runs(range_acc *a, u128 n, uint32_t k) {
  u128 x = n, E = n;
  for (uint32_t j = 0; j < k; j++) {
    if (x & 1) {
      if (x > (U128_MAX - 1) / 3) goto wide;
      x = x + (x >> 1) + 1;
      if (x > E) E = x;
    } else {
      x >>= 1;
    }
  }
  {
    u128 v = x + 1;
    uint64_t st = k;
    for (;;) {
      unsigned oa = ctz32((uint32_t)v | (1u << 8));
      u128 q = v >> oa;
      if (q > U128_MAX / P3[oa]) goto wide;
      v = q * P3[oa];
      st += oa;
      a->odd_runs++;
      if (v - 1 > E) E = v - 1;
      u128 m = v - 1;
      unsigned b = ctz32((uint32_t)m | 0x80000000u);
      a->even_runs++;
      if ((m >> b) < n) {
        unsigned i = 1;
        while ((m >> i) >= n) i++;
        st += i;
        break;
      }
      st += b;
      v = (m >> b) + 1;
    }
    big Eb;
    big_from_u128(&Eb, E);
    a->steps += st;
    acc_seed(a, n, st, &Eb);
    return;
  }
wide : {
  big nb, Eb;
  big_from_u128(&nb, n);
  uint64_t st2;
  if (big_seed(&nb, &st2, &Eb, &a->steps)) {
    a->failures++;
    return;
  }
  acc_seed(a, n, st2, &Eb);
}
}

/* ---- negative variant: m stands for -m, T'(m) = (3m-1)/2 (odd m), m/2
 * (even m), which is T acting on -m.  sigma and E as for T.  A seed that
 * returns to itself lies on a cycle and never descends (in range: the cycle
 * minima 5 and 17); it counts as a failure, as does one that reaches the
 * step cap or leaves 512 bits. */

static void neg_wide(range_acc *a, u128 n) {
  big nb, Eb;
  big_from_u128(&nb, n);
  uint64_t st2;
  if (big_seed_v(&nb, &st2, &Eb, &a->steps, 1)) {
    a->failures++;
    return;
  }
  acc_seed(a, n, st2, &Eb);
}

/* method 0: single T'-steps in u128 */
static void seed_steps_neg(range_acc *a, u128 n) {
  u128 x = n, E = n;
  uint64_t st = 0;
  for (;;) {
    if (x & 1) {
      if (x > U128_MAX - (x >> 1)) {
        neg_wide(a, n);
        return;
      }
      x = x + (x >> 1);
      if (x > E) E = x;
    } else {
      x >>= 1;
    }
    st++;
    if (x < n) break;
    if (x == n || st >= NEG_STEP_CAP) {
      a->failures++;
      return;
    }
  }
  big Eb;
  big_from_u128(&Eb, E);
  a->steps += st;
  acc_seed(a, n, st, &Eb);
}

/* the run-length loop in the "-1" space, u = T'^k(m) - 1: odd run
 * a = ctz(u | 2^8), u = 3^a (u >> a); even run b = ctz((u+1) | 2^31),
 * u = ((u+1) >> b) - 1.  Descent happens inside an even run; a return to
 * the seed happens at the end of one.  Starts from u after s steps. */
static void runs_neg(range_acc *a, u128 n, u128 u, uint64_t st, u128 E) {
  for (;;) {
    unsigned oa = ctz32((uint32_t)u | (1u << 8));
    u128 q = u >> oa;
    if (q > U128_MAX / P3[oa] || q * P3[oa] == U128_MAX) {
      neg_wide(a, n);
      return;
    }
    u = q * P3[oa];
    st += oa;
    a->odd_runs++;
    if (u + 1 > E) E = u + 1;
    u128 t = u + 1;
    unsigned b = ctz32((uint32_t)t | 0x80000000u);
    a->even_runs++;
    if ((t >> b) < n) {
      unsigned i = 1;
      while ((t >> i) >= n) i++;
      st += i;
      break;
    }
    st += b;
    if ((t >> b) == n || st >= NEG_STEP_CAP) {
      a->failures++;
      return;
    }
    u = (t >> b) - 1;
  }
  big Eb;
  big_from_u128(&Eb, E);
  a->steps += st;
  acc_seed(a, n, st, &Eb);
}

/* method 1 */
static void seed_runs_neg(range_acc *a, u128 n) { runs_neg(a, n, n - 1, 0, n); }

/* method 2: the first k steps as single steps (no descent for a survivor),
 * then the run-length loop */
static void seed_jump_runs_neg(range_acc *a, u128 n, uint32_t k) {
  u128 x = n, E = n;
  for (uint32_t j = 0; j < k; j++) {
    if (x & 1) {
      if (x > U128_MAX - (x >> 1)) {
        neg_wide(a, n);
        return;
      }
      x = x + (x >> 1);
      if (x > E) E = x;
    } else {
      x >>= 1;
    }
  }
  runs_neg(a, n, x - 1, k, E);
}

typedef struct {
  u128 lo, hi; /* [lo, hi) */
  uint32_t k;
  int use_mod9, method, neg;
  const uint8_t *bits;
  const uint8_t *pre; /* direct test: the 2^DIRECT_PREFILTER_K sieve, or NULL */
  range_acc acc;
} range_job;

static void *range_worker(void *p) {
  range_job *j = (range_job *)p;
  const u128 K = (u128)1 << j->k;
  const uint64_t mask = (j->k ? (1ull << j->k) - 1 : 0);
  for (u128 n = j->lo; n < j->hi; n++) {
    if (n < 2) continue;
    if (j->use_mod9) {
      unsigned r9 = (unsigned)(n % 9);
      /* T: keep {0,1,3,6,7} (cu:488).  T': m = 1 mod 3 (m > 1) is T' of the
       * smaller odd (2m+1)/3, and m = 5 mod 9 (m > 5) is T'^3 of the smaller
       * x = (8m+5)/9 (x = 5 mod 8: odd, odd, even steps); keep {0,2,3,6,8}. */
      if (j->neg ? !(((0x14Du >> r9) & 1) || n == 5) : !((0xCBu >> r9) & 1)) continue;
    }
    if (j->k && n >= K) {
      uint64_t r = (uint64_t)n & mask;
      if (j->bits) {
        if (!((j->bits[r >> 3] >> (r & 7)) & 1)) continue;
      } else {
        const uint64_t rp = r & ((1ull << DIRECT_PREFILTER_K) - 1);
        if (j->pre && !((j->pre[rp >> 3] >> (rp & 7)) & 1)) continue;
        if (!residue_survives_v(r, j->k, j->neg)) continue;
      }
    }
    j->acc.seeds++;
    if (j->neg) {
      if (j->method == 0)
        seed_steps_neg(&j->acc, n);
      else if (j->method == 2 && j->k && n >= K)
        seed_jump_runs_neg(&j->acc, n, j->k);
      else
        seed_runs_neg(&j->acc, n);
    } else if (j->method == 0) {
      seed_steps(&j->acc, n);
    } else if (j->method == 3) {
      seed_runs64(&j->acc, n);
    } else if (j->method == 2 && j->k && n >= K) {
      seed_jump_runs(&j->acc, n, j->k);
    } else {
      seed_runs(&j->acc, n);
    }
  }
  return NULL;
}

int orc_range(uint64_t offset_lo, uint64_t offset_hi, uint64_t size,
              uint32_t k, int use_mod9, int method, int nthreads,
              orc_range_result *out) {
  /* the table costs 2^k residue tests, the direct test k steps per seed */
  const int direct = k > 26 || (u128)size * k < ((u128)1 << k);
  return orc_range_ex(offset_lo, offset_hi, size, k, use_mod9, method, nthreads,
                      direct ? ORC_RANGE_DIRECT_SIEVE : 0, out);
}

int orc_range_ex(uint64_t offset_lo, uint64_t offset_hi, uint64_t size,
                 uint32_t k, int use_mod9, int method, int nthreads,
                 int flags, orc_range_result *out) {
  u128 offset = U128_OF(offset_lo, offset_hi);
  if (k > 34 || nthreads < 1) return -1;
  const int neg = (flags & ORC_RANGE_NEGATIVE) != 0;
  const int direct_sieve = neg || (flags & ORC_RANGE_DIRECT_SIEVE);
  memset(out, 0, sizeof *out);
  const uint8_t *bits = NULL, *pre = NULL;
  if (k && !direct_sieve) {
    bits = cached_sieve(k);
    if (!bits) return -2;
  } else if (k > DIRECT_PREFILTER_K && !neg) {
    pre = cached_sieve(DIRECT_PREFILTER_K);
  }
  range_job *jobs = (range_job *)calloc((size_t)nthreads, sizeof *jobs);
  pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof *th);
  uint64_t per = size / (uint64_t)nthreads, rem = size % (uint64_t)nthreads;
  u128 cur = offset;
  for (int i = 0; i < nthreads; i++) {
    uint64_t len = per + ((uint64_t)i < rem ? 1 : 0);
    jobs[i].lo = cur;
    jobs[i].hi = cur + len;
    cur += len;
    jobs[i].k = k;
    jobs[i].use_mod9 = use_mod9;
    jobs[i].method = method;
    jobs[i].neg = neg;
    jobs[i].bits = bits;
    jobs[i].pre = pre;
  }
  for (int i = 1; i < nthreads; i++) pthread_create(&th[i], NULL, range_worker, &jobs[i]);
  range_worker(&jobs[0]);
  for (int i = 1; i < nthreads; i++) pthread_join(th[i], NULL);
  range_acc tot;
  memset(&tot, 0, sizeof tot);
  for (int i = 0; i < nthreads; i++) acc_merge(&tot, &jobs[i].acc);
  out->seeds = tot.seeds;
  out->failures = tot.failures;
  out->steps = tot.steps;
  out->odd_runs = tot.odd_runs;
  out->even_runs = tot.even_runs;
  out->wide64 = tot.wide64;
  if (tot.have) {
    big_to_u32(&tot.E, out->max_exc);
    for (int i = 0; i < 4; i++) {
      out->max_exc_seed[i] = (uint32_t)(tot.E_seed >> (32 * i));
      out->max_st_seed[i] = (uint32_t)(tot.st_seed >> (32 * i));
    }
    out->max_st = tot.st;
  }
  free(jobs);
  free(th);
  return 0;
}

/* ===================================================================== */
/* Trajectory queries.                                                   */
/* ===================================================================== */

int orc_trajectory(const uint32_t *seeds, uint32_t nseeds, uint32_t seed_limbs,
                   uint64_t *st, uint32_t *exc, uint32_t *status) {
  if (seed_limbs == 0 || seed_limbs > 8) return -1;
  for (uint32_t i = 0; i < nseeds; i++) {
    big n, E;
    big_from_u32(&n, seeds + (size_t)i * seed_limbs, seed_limbs);
    int small = 1;
    for (int w = 1; w < 8; w++) small &= n.w[w] == 0;
    if (small && n.w[0] < 2) {
      st[i] = 0;
      big_to_u32(&n, exc + (size_t)i * 16);
      status[i] = 1;
      continue;
    }
    uint64_t s;
    int rc = big_seed(&n, &s, &E, NULL);
    if (rc) {
      st[i] = 0;
      memset(exc + (size_t)i * 16, 0, 64);
      status[i] = 2;
      continue;
    }
    st[i] = s;
    big_to_u32(&E, exc + (size_t)i * 16);
    status[i] = 0;
  }
  return 0;
}
