/*
 * ref_tool.cpp -- drives the reference's own functions (collatz_cudav7.cu
 * compiled for the CPU through ref_shim/cuda_runtime.h) on explicit
 * batches of Step-1 pairs, to make pair-level golden vectors.
 *
 * TEST INFRASTRUCTURE ONLY (built by oracle/build_ref.sh into oracle/_ref).
 *
 * stdin commands, one per line:
 *   T <path>                       write the 16 bit vectors and the mod-9
 *                                  sieve (u32 little-endian) to <path>
 *   K <bigindex> <n> <8n words>    run compute_kernel (cu:185-411) on the
 *                                  pairs; prints any overflow seeds the
 *                                  kernel prints, then "HASH <hex> <seeds>"
 *   S <bigindex> <base_lo> <base_hi> <number_lo> <number_hi>
 *                                  run search2 (cu:654-682) with
 *                                  threepower = THREEPOWEROFFSET+bigindex;
 *                                  prints overflow seeds, then "HASH <hex>"
 */
#define main ref_program_main
#include REF_SOURCE
#undef main

static PrecomputedData g_data;
static std::vector<u32> g_flat, g_flat9;

/* The table set-up that the reference's main() does inline (cu:104-171). */
static void ref_setup() {
  u128 a = 1;
  THREEPOWERS[0] = a;
  for (isize i = 1; i < 80; i++) {
    a *= 3;
    THREEPOWERS[i] = a;
  }
  for (auto &v : g_data.initialbitarray) v.resize(INITIALBITARRAYSIZE);
  for (auto &v : g_data.mod9sieve) v.resize(LASTBITSTEPS);
  u32 m = 1;
  for (isize i = 1; i < 128; i++) {
    m *= ONETHIRD;
    if (i >= THREEPOWEROFFSET && i - THREEPOWEROFFSET < 16) g_data.magicnumbers[i - THREEPOWEROFFSET] = m;
  }
  precompute(&g_data);
  g_flat.resize(16 * INITIALBITARRAYSIZE);
  for (int r = 0; r < 16; r++)
    std::memcpy(&g_flat[r * INITIALBITARRAYSIZE], g_data.initialbitarray[r].data(), INITIALBITARRAYSIZE * 4);
  g_flat9.resize(9 * LASTBITSTEPS);
  for (int r = 0; r < 9; r++) std::memcpy(&g_flat9[r * LASTBITSTEPS], g_data.mod9sieve[r].data(), LASTBITSTEPS * 4);
}

int main() {
  ref_setup();
  char cmd[8];
  while (std::scanf("%7s", cmd) == 1) {
    if (cmd[0] == 'T') {
      char path[4096];
      if (std::scanf("%4095s", path) != 1) return 2;
      FILE *f = std::fopen(path, "wb");
      if (!f) return 3;
      std::fwrite(g_flat.data(), 4, g_flat.size(), f);
      std::fwrite(g_flat9.data(), 4, g_flat9.size(), f);
      std::fclose(f);
      std::printf("TABLES %zu %zu\n", g_flat.size(), g_flat9.size());
    } else if (cmd[0] == 'K') {
      unsigned bigindex, n;
      if (std::scanf("%u %u", &bigindex, &n) != 2) return 2;
      std::vector<u32> pairs(8 * (size_t)n);
      for (auto &w : pairs)
        if (std::scanf("%u", &w) != 1) return 2;
      u32 hash[HASHTABLESIZE] = {};
      u128 tpv = THREEPOWERS[THREEPOWEROFFSET + bigindex];
      unsigned long long before = shim_seed_count;
      u32 blocks = (n + 255) / 256;
      SHIM_LAUNCH(blocks, 256, compute_kernel, g_flat.data(), g_flat9.data(), pairs.data(), bigindex, n,
                  g_data.magicnumbers[bigindex], (u32)tpv, (u32)(tpv >> 32), (u32)(tpv >> 64), (u32)(tpv >> 96),
                  hash);
      u32 h = 0;
      for (int i = 0; i < (int)HASHTABLESIZE; i++) h ^= hash[i];
      std::printf("HASH %X %llu\n", h, shim_seed_count - before);
    } else if (cmd[0] == 'S') {
      unsigned bigindex;
      unsigned long long blo, bhi, nlo, nhi;
      if (std::scanf("%u %llu %llu %llu %llu", &bigindex, &blo, &bhi, &nlo, &nhi) != 5) return 2;
      u128 base = ((u128)bhi << 64) | blo, number = ((u128)nhi << 64) | nlo;
      u32 h = search2(base, THREEPOWEROFFSET + bigindex, number, &g_data, bigindex);
      std::printf("HASH %X\n", h);
    }
    std::fflush(stdout);
  }
  return 0;
}
