// collatz_b200 -- drop-in for the reference program collatz_cudav7.cu.
//
//   echo "3 2 2 9 1 0" | collatz_b200 [N]
//
// Reads one 6-tuple "base sigfig threepower number doubleeven numevens" from
// stdin (cu:96-101), verifies all n < 2^N below that Step-1 node on the GPU,
// prints every seed whose trajectory reaches 2^100 on stdout in the
// reference's format (cu:298) and the reference's summary line on stderr
// (cu:181-182), followed by one "# results {...}" JSON line with the outputs
// the reference does not compute, the device time (device_ms) and the wall
// time of the run after the context and its tables exist (run_ms).  N
// defaults to 45 (MAXBITS, cu:43) or the
// COLLATZ_MAXBITS environment variable.
//
//   collatz_b200 --cases FILE [--journal JOURNAL] [N]
//
// runs every line of a cases_* file (one 6-tuple per line) in one process
// and prints the combined outputs in the same format: the overflow seeds of
// all lines, then the summary line with the summed launch count and the XOR
// of the lines' hashes (the hash of the whole tree).  With --journal, each
// finished line is recorded and a rerun resumes after the last finished one.
//
// Step 1 (search1, cu:497-563) runs on the GPU; --host-step1 runs it on the
// host threads instead (same outputs).
#include <chrono>
#include <cinttypes>
#include <fstream>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "collatz.h"

static std::string u128s(const uint32_t* w, int n) {
  unsigned __int128 x = 0;
  for (int i = n - 1; i >= 0; i--) x = (x << 32) | w[i];
  if (x == 0) return "0";
  std::string s;
  while (x) {
    s.insert(s.begin(), char('0' + (int)(x % 10)));
    x /= 10;
  }
  return s;
}

static collatz_case parse_case(const std::string& line, bool* ok) {
  std::istringstream iss(line);
  uint64_t a[6] = {0, 0, 0, 0, 0, 0};
  *ok = static_cast<bool>(iss >> a[0] >> a[1] >> a[2] >> a[3] >> a[4] >> a[5]);
  return collatz_case{{a[0], 0}, (uint32_t)a[1], (uint32_t)a[2], {a[3], 0}, (uint32_t)a[4], (uint32_t)a[5]};
}

int main(int argc, char** argv) {
  uint32_t maxbits = 45;
  if (const char* e = std::getenv("COLLATZ_MAXBITS")) maxbits = (uint32_t)std::atoi(e);
  std::string cases_file, journal;
  bool host_step1 = false;
  for (int i = 1; i < argc; i++) {
    const std::string a = argv[i];
    if (a == "--host-step1") {
      host_step1 = true;
    } else if (a == "--cases" && i + 1 < argc) {
      cases_file = argv[++i];
    } else if (a == "--journal" && i + 1 < argc) {
      journal = argv[++i];
    } else {
      maxbits = (uint32_t)std::atoi(argv[i]);
    }
  }
  std::vector<collatz_case> cases;
  if (!cases_file.empty()) {
    std::ifstream f(cases_file);
    if (!f) {
      std::fprintf(stderr, "cannot read %s\n", cases_file.c_str());
      return 2;
    }
    std::string line;
    while (std::getline(f, line)) {
      bool ok = false;
      const collatz_case c = parse_case(line, &ok);
      if (ok) cases.push_back(c);
    }
  } else {
    std::string line;
    std::getline(std::cin, line);
    bool ok = false;
    cases.push_back(parse_case(line, &ok));
  }

  collatz_config cfg;
  collatz_config_default(&cfg);
  cfg.maxbits = maxbits;
  if (host_step1) cfg.flags |= COLLATZ_CFG_HOST_STEP1;
  collatz_ctx* ctx = nullptr;
  int rc = collatz_create(&cfg, &ctx);
  if (rc) {
    std::fprintf(stderr, "collatz_create: %s\n", collatz_status_string(rc));
    return 2;
  }
  const uint64_t cap = 1u << 20;
  std::vector<uint32_t> ov(4 * cap);
  collatz_case_result r = {};
  r.overflow_seeds = ov.data();
  r.overflow_cap = cap;
  uint32_t n_run = 1;
  const auto t_run = std::chrono::steady_clock::now();  // after the context and tables exist
  if (cases_file.empty()) {
    rc = collatz_run_case(ctx, &cases[0], &r);
  } else {
    rc = collatz_run_cases(ctx, cases.data(), (uint32_t)cases.size(), journal.empty() ? nullptr : journal.c_str(),
                           nullptr, &r, &n_run);
  }
  const double run_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_run).count();
  if (rc && rc != COLLATZ_E_DEVICE) {
    std::fprintf(stderr, "collatz_run_case: %s: %s\n", collatz_status_string(rc), collatz_last_error(ctx));
    collatz_destroy(ctx);
    return 3;
  }
  for (uint64_t i = 0; i < r.n_overflow && i < cap; i++)
    std::printf("%X%08X%08X\n", ov[4 * i + 2], ov[4 * i + 1], ov[4 * i]);
  std::fflush(stdout);
  std::fprintf(stderr, "Number of kernel launches = %" PRIu64 ". ", r.launches);
  std::fprintf(stderr, "Spot checks = %u. Complete hash = %X.\n", r.spot_checks, r.hash);
  std::fprintf(stderr,
               "# results {\"seeds_checked\": %" PRIu64 ", \"pairs\": %" PRIu64 ", \"cpu_pairs\": %" PRIu64
               ", \"overflow\": %" PRIu64
               ", \"max_excursion\": \"%s\", \"max_excursion_seed\": \"%s\", \"max_stopping_time\": %" PRIu64
               ", \"max_stopping_time_seed\": \"%s\", \"errors\": %u, \"device_ms\": %.3f, \"run_ms\": %.3f"
               ", \"cases\": %zu, \"cases_run\": %u}\n",
               r.seeds_checked, r.pairs, r.cpu_pairs, r.n_overflow, u128s(r.max_excursion, 4).c_str(),
               u128s(r.max_excursion_seed, 4).c_str(), r.max_stopping_time, u128s(r.max_stopping_time_seed, 4).c_str(),
               r.errors, r.device_ms, run_ms, cases.size(), n_run);
  collatz_destroy(ctx);
  return r.errors ? 4 : 0;
}
