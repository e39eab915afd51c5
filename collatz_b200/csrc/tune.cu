// tune.cu -- autotuner for the kernel variants (collatz_autotune).
//
// The range kernel comes in variants of block shape (run pairs between
// refills R, minimum resident blocks per SM), the cases kernel in variants of
// checkpoints per pass and refill threshold.  The autotuner times every
// variant of a mode on a fixed sample on this device, keeps the fastest for
// the context, and records it in a small text cache keyed by the device, the
// library's variant set and the workload parameter (range: sieve exponent k;
// cases: N), so that later contexts created with COLLATZ_VARIANT_AUTO pick it
// up without timing again.  Results never depend on the variant: every
// variant computes the same outputs (the tests check each one).
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "runtime.h"

using namespace cz;

namespace {

std::string device_key(const collatz_ctx* c) {
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, c->device) != cudaSuccess) {
    cudaGetLastError();
    return "";
  }
  std::string name = p.name;
  for (char& ch : name)
    if (ch == ' ' || ch == '\t') ch = '_';
  std::ostringstream k;
  k << name << ":sm" << p.multiProcessorCount << ":cc" << p.major << "." << p.minor << ":abi"
    << COLLATZ_ABI_VERSION << ":v" << range_variants() << "." << cases_variants() << "." << range64_variants()
    << "." << std::hex << range64_variant_rev();
  return k.str();
}

std::string cache_path() {
  if (const char* e = getenv("COLLATZ_TUNE_CACHE")) return e;
  if (const char* x = getenv("XDG_CACHE_HOME")) return std::string(x) + "/collatz_b200/tune.txt";
  if (const char* h = getenv("HOME")) return std::string(h) + "/.cache/collatz_b200/tune.txt";
  return "";
}

// Cache lines: "<mode> <device key> <param> <variant> <ms per variant ...>"
bool cache_lookup(const std::string& path, const char* mode, const std::string& key, uint32_t param,
                  int nvariants, int* variant) {
  if (path.empty() || key.empty()) return false;
  std::ifstream f(path);
  std::string line;
  bool found = false;
  while (std::getline(f, line)) {
    std::istringstream s(line);
    std::string m, k;
    uint32_t pa = 0;
    int v = -1;
    if (!(s >> m >> k >> pa >> v)) continue;
    if (m == mode && k == key && pa == param && v >= 0 && v < nvariants) {
      *variant = v;  // the last matching line wins
      found = true;
    }
  }
  return found;
}

void mkdirs(const std::string& path) {
  for (size_t i = 1; i < path.size(); i++)
    if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
}

void cache_store(const std::string& path, const char* mode, const std::string& key, uint32_t param, int variant,
                 const float* ms, int n) {
  if (path.empty() || key.empty()) return;
  std::vector<std::string> keep;
  {
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
      std::istringstream s(line);
      std::string m, k;
      uint32_t pa = 0;
      if ((s >> m >> k >> pa) && m == mode && k == key && pa == param) continue;
      if (!line.empty()) keep.push_back(line);
    }
  }
  std::ostringstream nl;
  nl << mode << " " << key << " " << param << " " << variant;
  for (int i = 0; i < n; i++) nl << " " << ms[i];
  keep.push_back(nl.str());
  mkdirs(path);
  const std::string tmp = path + ".tmp" + std::to_string((long)getpid());
  {
    std::ofstream f(tmp);
    for (const std::string& l : keep) f << l << "\n";
    if (!f) return;
  }
  std::rename(tmp.c_str(), path.c_str());
}

float median3(float a, float b, float c) { return std::max(std::min(a, b), std::min(std::max(a, b), c)); }

// Device time of one plan launch over the range sample, median of 3 after a warm-up.
int time_range(collatz_ctx* c, const collatz_range& r, float* ms) {
  collatz_plan* p = nullptr;
  int rc = collatz_plan_create(c, &r, 1, &p);
  if (rc) return rc;
  float t[4];
  collatz_range_result res;
  for (int i = 0; i < 4 && !rc; i++) {
    rc = collatz_plan_launch(p);
    if (!rc) rc = collatz_plan_results(p, &res);
    t[i] = (float)res.device_ms;
  }
  collatz_plan_destroy(p);
  if (!rc) *ms = median3(t[1], t[2], t[3]);
  return rc;
}

int time_cases(collatz_ctx* c, uint32_t bigindex, const std::vector<uint32_t>& pairs, float* ms) {
  collatz_case_result res;
  float t[4];
  for (int i = 0; i < 4; i++) {
    std::memset(&res, 0, sizeof res);
    const int rc = collatz_verify_pairs(c, bigindex, pairs.data(), (uint32_t)(pairs.size() / 8), &res);
    if (rc) return rc;
    t[i] = (float)res.device_ms;
  }
  *ms = median3(t[1], t[2], t[3]);
  return COLLATZ_OK;
}

// Step-1 leaves of the reference's root case (3 2 2 9 1 0) for this N, taken
// subtree by subtree until about 2^20 pairs; returns the fullest bucket.
void cases_sample(const collatz_ctx* c, uint32_t* bigindex, std::vector<uint32_t>& out) {
  const uint32_t mbi = c->ct.mbi, tpo = c->ct.tpo;
  Step1 s1(mbi, tpo);
  Step1Node root{3, 2, 2, 9, 1, 0};
  std::vector<Step1Node> roots;
  s1.split(root, std::min<uint32_t>(mbi, 12), roots);
  std::vector<std::vector<uint32_t>> buckets(16);
  size_t total = 0;
  for (const Step1Node& r : roots) {
    s1.leaves(r, [&](uint32_t bi, u128 b, u128 num) {
      if (bi >= 16) return;
      uint32_t w[8];
      pack_pair(w, b, num, bi);
      buckets[bi].insert(buckets[bi].end(), w, w + 8);
      total++;
    });
    if (total >= (1u << 20)) break;
  }
  size_t best = 0;
  for (uint32_t i = 1; i < 16; i++)
    if (buckets[i].size() > buckets[best].size()) best = i;
  *bigindex = (uint32_t)best;
  out.swap(buckets[best]);
}

}  // namespace

namespace cz {

// Applies cached choices to a new context (COLLATZ_VARIANT_AUTO); with
// COLLATZ_AUTOTUNE=1 in the environment, tunes what the cache lacks.
void tune_on_create(collatz_ctx* c) {
  const std::string key = device_key(c), path = cache_path();
  int v = -1;
  bool have_r = false, have_c = false;
  if (cache_lookup(path, "range", key, c->cfg.range_k, range_variants(), &v)) {
    c->range_variant = v;
    have_r = true;
    if (cache_lookup(path, "range64", key, c->cfg.range_k, range64_variants(), &v)) c->range64_variant = v;
    else have_r = false;
    if (cache_lookup(path, "range64bits", key, c->cfg.range_k, (int)range64_max_seed_bits() + 1, &v))
      c->range64_bits = (uint32_t)v;
    else have_r = false;
  }
  if (cache_lookup(path, "cases", key, c->cfg.maxbits, cases_variants(), &v)) {
    c->cases_variant = v;
    have_c = true;
  }
  const char* e = getenv("COLLATZ_AUTOTUNE");
  if (e && e[0] == '1' && (!have_r || !have_c)) {
    collatz_tune_result r;
    collatz_autotune(c, (have_r ? 0u : COLLATZ_TUNE_RANGE) | (have_c ? 0u : COLLATZ_TUNE_CASES), &r);
  }
}

}  // namespace cz

extern "C" int collatz_autotune(collatz_ctx* c, uint32_t flags, collatz_tune_result* out) {
  if (!c) return COLLATZ_E_ARG;
  std::lock_guard<std::recursive_mutex> g(c->mu);
  DeviceScope dev_scope(c->device);
  if (dev_scope.err != cudaSuccess) return set_cuda_error(c, dev_scope.err, "collatz_autotune");
  collatz_tune_result res;
  std::memset(&res, 0, sizeof res);
  for (int i = 0; i < 8; i++) res.range_ms[i] = res.cases_ms[i] = res.range64_ms[i] = -1.0f;
  for (int i = 0; i < 4; i++) res.width_ms[i] = -1.0f;
  res.range_variant = c->range_variant;
  res.cases_variant = c->cases_variant;
  res.range64_variant = c->range64_variant;
  res.range64_bits = c->range64_bits;
  const std::string key = device_key(c), path = (flags & COLLATZ_TUNE_NO_CACHE) ? "" : cache_path();
  int rc = COLLATZ_OK;
  if (flags & COLLATZ_TUNE_RANGE) {
    // sample: 2^34 seeds at 2^40 (aligned) with the context's default k
    collatz_range r{};
    r.offset[0] = 1ull << 40;
    r.size = 1ull << 34;
    r.k = c->cfg.range_k;
    const int keep = c->range_variant, keep64 = c->range64_variant;
    const uint32_t keep_bits = c->range64_bits;
    const int nv = std::min(range_variants(), 8), nv64 = std::min(range64_variants(), 8);
    c->range64_bits = 0;  // the four-limb kernel's variants
    for (int v = 0; v < nv && !rc; v++) {
      c->range_variant = v;
      rc = time_range(c, r, &res.range_ms[v]);
    }
    const int best = rc ? keep : (int)(std::min_element(res.range_ms, res.range_ms + nv) - res.range_ms);
    c->range_variant = best;
    c->range64_bits = range64_max_seed_bits();  // the 64-bit kernel's variants
    for (int v = 0; v < nv64 && !rc; v++) {
      c->range64_variant = v;
      rc = time_range(c, r, &res.range64_ms[v]);
    }
    const int best64 =
        rc ? keep64 : (int)(std::min_element(res.range64_ms, res.range64_ms + nv64) - res.range64_ms);
    c->range64_variant = best64;
    // limb width: both kernels on seeds of 44 and of 48 bits
    uint32_t bits = 0;
    const uint32_t at_bits[2] = {44, range64_max_seed_bits()};
    for (int i = 0; i < 2 && !rc; i++) {
      collatz_range w = r;
      w.size = 1ull << 32;
      w.offset[0] = (1ull << at_bits[i]) - w.size;  // seeds of exactly at_bits[i] bits
      c->range64_bits = 0;
      rc = time_range(c, w, &res.width_ms[2 * i]);
      c->range64_bits = range64_max_seed_bits();
      if (!rc) rc = time_range(c, w, &res.width_ms[2 * i + 1]);
      if (!rc && res.width_ms[2 * i + 1] < res.width_ms[2 * i]) bits = at_bits[i];
    }
    if (!rc) {
      c->range64_bits = bits;
      res.range_variant = best;
      res.range64_variant = best64;
      res.range64_bits = bits;
      cache_store(path, "range", key, c->cfg.range_k, best, res.range_ms, nv);
      cache_store(path, "range64", key, c->cfg.range_k, best64, res.range64_ms, nv64);
      cache_store(path, "range64bits", key, c->cfg.range_k, (int)bits, res.width_ms, 4);
    } else {
      c->range_variant = keep;
      c->range64_variant = keep64;
      c->range64_bits = keep_bits;
    }
  }
  if (!rc && (flags & COLLATZ_TUNE_CASES)) {
    uint32_t bi = 0;
    std::vector<uint32_t> pairs;
    cases_sample(c, &bi, pairs);
    const int keep = c->cases_variant, nv = std::min(cases_variants(), 8);
    if (pairs.empty()) {
      res.cases_variant = keep;
    } else {
      for (int v = 0; v < nv && !rc; v++) {
        c->cases_variant = v;
        rc = time_cases(c, bi, pairs, &res.cases_ms[v]);
      }
      if (!rc) {
        const int best = (int)(std::min_element(res.cases_ms, res.cases_ms + nv) - res.cases_ms);
        c->cases_variant = best;
        res.cases_variant = best;
        cache_store(path, "cases", key, c->cfg.maxbits, best, res.cases_ms, nv);
      } else {
        c->cases_variant = keep;
      }
    }
  }
  if (out) *out = res;
  return rc;
}
