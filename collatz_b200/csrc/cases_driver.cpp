// cases_driver.cpp -- many cases_* lines in one process with a resume
// journal (collatz_run_cases, collatz_journal_load,
// collatz_combine_case_results).
//
// The reference verifies a bound 2^N by running its program once per line
// of a cases_* file (one Step-1 subtree root each) and combining the
// per-line outputs: the complete hash of the whole tree is the XOR of the
// lines' hashes (every checkpoint XOR lands in exactly one subtree), counts
// add up, and the overflow lists concatenate.  Here the lines run on one
// context in groups of up to 8192, each group as one device pass
// (collatz_run_case_batch: Step 1 from all the group's roots at once, one
// record per line), so the thousands of small lines of a cases_big file do
// not each pay a pass's fixed cost.  The group's lines are appended to a
// text journal and synced to disk before the next group starts, so a run
// that stops (a crash, a preempted job) resumes from the journal without
// repeating finished lines.
//
// Journal line (one per finished case, whitespace-separated):
//   case <index> <base lo> <base hi> <sigfig> <threepower> <number lo>
//        <number hi> <doubleeven> <numevens> <hash> <seeds> <launches>
//        <pairs> <cpu pairs> <n overflow> <E limbs 0..3> <E seed limbs 0..3>
//        <max sigma> <sigma seed limbs 0..3> <errors> <device ms>
//        <overflow seeds listed> <4 limbs each ...> end
// A line without the final "end" (a write cut short) is ignored.
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "collatz.h"

namespace {

constexpr uint64_t OV_CAP = 1u << 16;  // overflow seeds kept per case (and per group)
constexpr uint32_t GROUP = 8192;        // lines per device pass

bool less4(const uint32_t* a, const uint32_t* b) {
  for (int i = 3; i >= 0; i--)
    if (a[i] != b[i]) return a[i] < b[i];
  return false;
}

bool zero4(const uint32_t* a) { return (a[0] | a[1] | a[2] | a[3]) == 0; }

bool same_case(const collatz_case& a, const collatz_case& b) {
  return a.base[0] == b.base[0] && a.base[1] == b.base[1] && a.sigfig == b.sigfig &&
         a.threepower == b.threepower && a.number[0] == b.number[0] && a.number[1] == b.number[1] &&
         a.doubleeven == b.doubleeven && a.numevens == b.numevens;
}

std::string journal_line(uint32_t idx, const collatz_case& c, const collatz_case_result& r,
                         const uint32_t* ov, uint64_t nov) {
  std::ostringstream s;
  s << "case " << idx << " " << c.base[0] << " " << c.base[1] << " " << c.sigfig << " " << c.threepower << " "
    << c.number[0] << " " << c.number[1] << " " << c.doubleeven << " " << c.numevens << " " << r.hash << " "
    << r.seeds_checked << " " << r.launches << " " << r.pairs << " " << r.cpu_pairs << " " << r.n_overflow;
  for (int i = 0; i < 4; i++) s << " " << r.max_excursion[i];
  for (int i = 0; i < 4; i++) s << " " << r.max_excursion_seed[i];
  s << " " << r.max_stopping_time;
  for (int i = 0; i < 4; i++) s << " " << r.max_stopping_time_seed[i];
  char ms[32];
  std::snprintf(ms, sizeof ms, "%.6f", r.device_ms);
  s << " " << r.errors << " " << ms << " " << nov;
  for (uint64_t i = 0; i < 4 * nov; i++) s << " " << ov[i];
  s << " end\n";
  return s.str();
}

// Parses one journal line; false if malformed or cut short.
bool parse_line(const std::string& line, uint32_t* idx, collatz_case* c, collatz_case_result* r,
                std::vector<uint32_t>* ov) {
  std::istringstream s(line);
  std::string tag;
  if (!(s >> tag) || tag != "case") return false;
  std::memset(c, 0, sizeof *c);
  std::memset(r, 0, sizeof *r);
  uint64_t nov = 0;
  if (!(s >> *idx >> c->base[0] >> c->base[1] >> c->sigfig >> c->threepower >> c->number[0] >> c->number[1] >>
        c->doubleeven >> c->numevens >> r->hash >> r->seeds_checked >> r->launches >> r->pairs >> r->cpu_pairs >>
        r->n_overflow))
    return false;
  for (int i = 0; i < 4; i++) s >> r->max_excursion[i];
  for (int i = 0; i < 4; i++) s >> r->max_excursion_seed[i];
  s >> r->max_stopping_time;
  for (int i = 0; i < 4; i++) s >> r->max_stopping_time_seed[i];
  s >> r->errors >> r->device_ms >> nov;
  if (!s || nov > OV_CAP) return false;
  ov->resize(4 * nov);
  for (uint64_t i = 0; i < 4 * nov; i++) s >> (*ov)[i];
  std::string end;
  return (s >> end) && end == "end";
}

// Reads the journal into per-index results; returns COLLATZ_E_STATE when a
// recorded tuple differs from the case at its index.
int load(const char* path, const collatz_case* cases, uint32_t n, std::vector<collatz_case_result>& res,
         std::vector<std::vector<uint32_t>>& ovs, std::vector<uint8_t>& done) {
  res.assign(n, collatz_case_result{});
  ovs.assign(n, {});
  done.assign(n, 0);
  if (!path || !*path) return COLLATZ_OK;
  std::ifstream f(path);
  if (!f) return COLLATZ_OK;  // no journal yet
  std::string line;
  while (std::getline(f, line)) {
    uint32_t idx = 0;
    collatz_case c;
    collatz_case_result r;
    std::vector<uint32_t> ov;
    if (!parse_line(line, &idx, &c, &r, &ov)) continue;
    if (idx >= n || !same_case(c, cases[idx])) return COLLATZ_E_STATE;
    res[idx] = r;
    ovs[idx].swap(ov);
    done[idx] = 1;
  }
  return COLLATZ_OK;
}

int append(const char* path, const std::string& line) {
  FILE* f = std::fopen(path, "a");
  if (!f) return COLLATZ_E_ARG;
  const bool ok = std::fwrite(line.data(), 1, line.size(), f) == line.size() && std::fflush(f) == 0 &&
                  fsync(fileno(f)) == 0;
  std::fclose(f);
  return ok ? COLLATZ_OK : COLLATZ_E_ARG;
}

}  // namespace

extern "C" int collatz_combine_case_results(const collatz_case_result* parts, uint32_t n, collatz_case_result* out) {
  if (!out || (n && !parts)) return COLLATZ_E_ARG;
  uint32_t* ovbuf = out->overflow_seeds;
  const uint64_t ovcap = out->overflow_cap;
  std::memset(out, 0, sizeof *out);
  out->overflow_seeds = ovbuf;
  out->overflow_cap = ovcap;
  std::vector<uint32_t> ov;
  bool have_e = false, have_s = false;
  for (uint32_t i = 0; i < n; i++) {
    const collatz_case_result& p = parts[i];
    out->hash ^= p.hash;
    out->spot_checks += p.spot_checks;
    out->launches += p.launches;
    out->seeds_checked += p.seeds_checked;
    out->pairs += p.pairs;
    out->cpu_pairs += p.cpu_pairs;
    out->n_overflow += p.n_overflow;
    out->errors |= p.errors;
    out->device_ms += p.device_ms;
    if (p.overflow_seeds)
      ov.insert(ov.end(), p.overflow_seeds, p.overflow_seeds + 4 * std::min(p.n_overflow, p.overflow_cap));
    if (!zero4(p.max_excursion) &&
        (!have_e || less4(out->max_excursion, p.max_excursion) ||
         (!less4(p.max_excursion, out->max_excursion) && less4(p.max_excursion_seed, out->max_excursion_seed)))) {
      std::memcpy(out->max_excursion, p.max_excursion, sizeof p.max_excursion);
      std::memcpy(out->max_excursion_seed, p.max_excursion_seed, sizeof p.max_excursion_seed);
      have_e = true;
    }
    if (!zero4(p.max_stopping_time_seed) &&
        (!have_s || p.max_stopping_time > out->max_stopping_time ||
         (p.max_stopping_time == out->max_stopping_time &&
          less4(p.max_stopping_time_seed, out->max_stopping_time_seed)))) {
      out->max_stopping_time = p.max_stopping_time;
      std::memcpy(out->max_stopping_time_seed, p.max_stopping_time_seed, sizeof p.max_stopping_time_seed);
      have_s = true;
    }
  }
  // overflow seeds sorted ascending, as collatz_run_case reports them
  const size_t m = ov.size() / 4;
  std::vector<uint32_t> order(m);
  for (size_t i = 0; i < m; i++) order[i] = (uint32_t)i;
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return less4(&ov[4 * a], &ov[4 * b]); });
  if (ovbuf)
    for (size_t i = 0; i < m && i < ovcap; i++) std::memcpy(ovbuf + 4 * i, &ov[4 * order[i]], 16);
  return COLLATZ_OK;
}

extern "C" int collatz_journal_load(const char* journal, const collatz_case* cases, uint32_t n,
                                    collatz_case_result* results, uint8_t* done) {
  if (!journal || (n && (!cases || !results || !done))) return COLLATZ_E_ARG;
  std::vector<collatz_case_result> res;
  std::vector<std::vector<uint32_t>> ovs;
  std::vector<uint8_t> dn;
  const int rc = load(journal, cases, n, res, ovs, dn);
  if (rc) return rc;
  for (uint32_t i = 0; i < n; i++) {
    done[i] = dn[i];
    if (!dn[i]) continue;
    uint32_t* buf = results[i].overflow_seeds;
    const uint64_t cap = results[i].overflow_cap;
    results[i] = res[i];
    results[i].overflow_seeds = buf;
    results[i].overflow_cap = cap;
    if (buf)
      for (size_t j = 0; j < ovs[i].size() / 4 && j < cap; j++) std::memcpy(buf + 4 * j, &ovs[i][4 * j], 16);
  }
  return COLLATZ_OK;
}

extern "C" int collatz_run_cases(collatz_ctx* ctx, const collatz_case* cases, uint32_t n, const char* journal,
                                 collatz_case_result* per_case, collatz_case_result* combined, uint32_t* n_run) {
  if (!ctx || !combined || (n && !cases)) return COLLATZ_E_ARG;
  std::vector<collatz_case_result> res;
  std::vector<std::vector<uint32_t>> ovs;
  std::vector<uint8_t> done;
  int rc = load(journal, cases, n, res, ovs, done);
  if (rc) return rc;
  uint32_t ran = 0;
  std::vector<uint32_t> todo;
  for (uint32_t i = 0; i < n; i++)
    if (!done[i]) todo.push_back(i);
  std::vector<uint32_t> pool(4 * OV_CAP);
  std::vector<collatz_case> gc;
  std::vector<collatz_case_result> gr;
  for (size_t g0 = 0; g0 < todo.size(); g0 += GROUP) {
    const uint32_t m = (uint32_t)std::min<size_t>(GROUP, todo.size() - g0);
    gc.resize(m);
    gr.resize(m);
    for (uint32_t j = 0; j < m; j++) gc[j] = cases[todo[g0 + j]];
    rc = collatz_run_case_batch(ctx, gc.data(), m, gr.data(), pool.data(), OV_CAP);
    if (rc && rc != COLLATZ_E_DEVICE) return rc;  // a device error bit is recorded in the line's errors
    std::string text;
    for (uint32_t j = 0; j < m; j++) {
      const uint32_t i = todo[g0 + j];
      const collatz_case_result& r = gr[j];
      const uint64_t nov = r.overflow_seeds ? r.overflow_cap : 0;
      ovs[i].assign(r.overflow_seeds, r.overflow_seeds + 4 * nov);
      if (journal && *journal) text += journal_line(i, cases[i], r, ovs[i].data(), nov);
      res[i] = r;
      done[i] = 1;
      ran++;
    }
    if (journal && *journal) {
      const int wrc = append(journal, text);
      if (wrc) return wrc;
    }
  }
  for (uint32_t i = 0; i < n; i++) {
    res[i].overflow_seeds = ovs[i].empty() ? nullptr : ovs[i].data();
    res[i].overflow_cap = ovs[i].size() / 4;
  }
  rc = collatz_combine_case_results(res.data(), n, combined);
  if (per_case)
    for (uint32_t i = 0; i < n; i++) {
      per_case[i] = res[i];
      per_case[i].overflow_seeds = nullptr;
      per_case[i].overflow_cap = 0;
    }
  if (n_run) *n_run = ran;
  if (!rc && combined->errors) rc = COLLATZ_E_DEVICE;
  return rc;
}
