// Command-line front end of the CPU restatement (test infrastructure only).
//   csm_oracle -q query.graph -d data(.graph|.bin) -u stream(.txt|.bin)
//              [--max-results N] [--homo 0|1] [--no-hash] [--max-updates N]
//              [--out per_update.csv]
// Writes the same per-update CSV columns as oracle/ref_build/ref_driver.cpp
// plus the canonical algorithmic bytes and the status.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "csm_oracle.h"

namespace {

bool slurp(const std::string& p, std::string& b) {
  FILE* f = fopen(p.c_str(), "rb");
  if (!f) return false;
  fseek(f, 0, SEEK_END); long n = ftell(f); fseek(f, 0, SEEK_SET);
  b.resize(n > 0 ? (size_t)n : 0);
  size_t got = n > 0 ? fread(&b[0], 1, (size_t)n, f) : 0;
  fclose(f);
  return got == b.size();
}

struct Words {
  const char* p; const char* e;
  bool next(std::string& w) {
    while (p < e && (unsigned char)*p <= ' ') p++;
    if (p >= e) return false;
    const char* s = p;
    while (p < e && (unsigned char)*p > ' ') p++;
    w.assign(s, (size_t)(p - s));
    return true;
  }
  uint32_t u() { std::string w; next(w); return (uint32_t)strtoul(w.c_str(), nullptr, 10); }
};

// Text graph (ParaCOSM/CSM/graph/graph.cpp:217-249) or "CSMG" binary.
bool load_graph(const std::string& p, std::vector<uint32_t>& vl, std::vector<uint32_t>& e) {
  std::string b;
  if (!slurp(p, b)) return false;
  vl.clear(); e.clear();
  if (b.size() >= 28 && memcmp(b.data(), "CSMG", 4) == 0) {
    uint32_t n; uint64_t m;
    memcpy(&n, b.data() + 8, 4); memcpy(&m, b.data() + 12, 8);
    vl.resize(n); e.resize(3 * m);
    memcpy(vl.data(), b.data() + 28, 4ULL * n);
    memcpy(e.data(), b.data() + 28 + 4ULL * n, 12ULL * m);
    return true;
  }
  Words w{b.data(), b.data() + b.size()};
  std::string t;
  while (w.next(t)) {
    if (t[0] == 't') { std::string x; w.next(x); w.next(x); continue; }
    if (t == "v") {
      uint32_t id = w.u(), l = w.u();
      if (id >= vl.size()) vl.resize((size_t)id + 1, 0xffffffffu);
      if (vl[id] == 0xffffffffu) vl[id] = l;
      continue;
    }
    uint32_t a = w.u(), c = w.u(), l = w.u();
    e.push_back(a); e.push_back(c); e.push_back(l);
  }
  return true;
}

// Text stream (graph.cpp:251-285) or "CSMU" binary.
bool load_stream(const std::string& p, std::vector<oracle_update>& s) {
  std::string b;
  if (!slurp(p, b)) return false;
  s.clear();
  if (b.size() >= 16 && memcmp(b.data(), "CSMU", 4) == 0) {
    uint64_t n; memcpy(&n, b.data() + 8, 8);
    s.resize(n);
    for (uint64_t i = 0; i < n; i++) {
      uint32_t r[4]; memcpy(r, b.data() + 16 + 16 * i, 16);
      oracle_update u{};
      u.type = (uint8_t)(r[0] & 0xff); u.is_add = (uint8_t)((r[0] >> 8) & 0xff);
      u.id1 = r[1]; u.id2 = r[2]; u.label = r[3];
      s[i] = u;
    }
    return true;
  }
  Words w{b.data(), b.data() + b.size()};
  std::string t;
  while (w.next(t)) {
    oracle_update u{};
    if (t == "v" || t == "-v") { u.type = 'v'; u.is_add = t == "v"; u.id1 = w.u(); u.label = w.u(); }
    else { u.type = 'e'; u.is_add = t == "e"; u.id1 = w.u(); u.id2 = w.u(); u.label = w.u(); }
    s.push_back(u);
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  std::string qp, dp, up, out;
  uint64_t maxr = 0, maxu = ~0ULL;
  int homo = 0, hash = 1;
  for (int i = 1; i < argc; i++) {
    std::string k = argv[i];
    auto nxt = [&]() -> std::string { if (i + 1 >= argc) exit(2); return argv[++i]; };
    if (k == "-q") qp = nxt(); else if (k == "-d") dp = nxt(); else if (k == "-u") up = nxt();
    else if (k == "--max-results") maxr = std::stoull(nxt());
    else if (k == "--homo") homo = std::stoi(nxt());
    else if (k == "--no-hash") hash = 0;
    else if (k == "--max-updates") maxu = std::stoull(nxt());
    else if (k == "--out") out = nxt();
    else { fprintf(stderr, "unknown flag %s\n", k.c_str()); return 2; }
  }
  std::vector<uint32_t> qvl, qe, vl, e;
  std::vector<oracle_update> s;
  if (!load_graph(qp, qvl, qe) || !load_graph(dp, vl, e) || !load_stream(up, s)) {
    fprintf(stderr, "cannot read inputs\n");
    return 1;
  }
  if (s.size() > maxu) s.resize(maxu);
  std::vector<oracle_result> r(s.size());
  auto t0 = std::chrono::steady_clock::now();
  int rc = oracle_run((uint32_t)qvl.size(), qvl.data(), (uint32_t)(qe.size() / 3), qe.data(), (uint32_t)vl.size(),
                      vl.data(), e.size() / 3, e.data(), s.size(), s.data(), maxr, homo, hash, r.data());
  auto t1 = std::chrono::steady_clock::now();
  if (rc != 0) { fprintf(stderr, "oracle_run failed %d\n", rc); return 1; }
  uint64_t pos = 0, neg = 0, bytes = 0, unsafe = 0;
  FILE* f = out.empty() ? nullptr : fopen(out.c_str(), "w");
  if (f) fprintf(f, "idx,type,is_add,id1,id2,label,pos,neg,hash,bytes,status\n");
  for (size_t i = 0; i < s.size(); i++) {
    pos += r[i].pos; neg += r[i].neg; bytes += r[i].bytes;
    if (r[i].pos || r[i].neg) unsafe++;
    if (f) fprintf(f, "%zu,%c,%d,%u,%u,%u,%llu,%llu,%llu,%llu,%u\n", i, s[i].type, s[i].is_add, s[i].id1, s[i].id2,
                   s[i].label, (unsigned long long)r[i].pos, (unsigned long long)r[i].neg,
                   (unsigned long long)r[i].hash, (unsigned long long)r[i].bytes, r[i].status);
  }
  if (f) fclose(f);
  printf("Incremental Matching: %.3f ms\n", std::chrono::duration<double, std::milli>(t1 - t0).count());
  printf("%zu edge updates.\n%llu unsafe updates.\n%llu positive matches.\n%llu negative matches.\n", s.size(),
         (unsigned long long)unsafe, (unsigned long long)pos, (unsigned long long)neg);
  printf("algorithmic_bytes=%llu\n", (unsigned long long)bytes);
  return 0;
}
