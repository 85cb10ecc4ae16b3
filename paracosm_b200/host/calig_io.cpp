#include "calig_io.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_set>

namespace csm {
namespace {

uint64_t edge_key(uint32_t a, uint32_t b) { return ((uint64_t)std::min(a, b) << 32) | std::max(a, b); }

bool slurp(const std::string& path, std::string& buf) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  fseek(f, 0, SEEK_END);
  const long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  buf.resize(sz > 0 ? (size_t)sz : 0);
  const size_t got = sz > 0 ? fread(&buf[0], 1, (size_t)sz, f) : 0;
  fclose(f);
  return got == buf.size();
}

// Whitespace-separated tokens of a whole file: words and signed integers.
struct Scan {
  const char* p;
  const char* e;
  bool skip() {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
    return p < e;
  }
  bool word(std::string& w) {
    if (!skip()) return false;
    const char* s = p;
    while (p < e && !(*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
    w.assign(s, (size_t)(p - s));
    return true;
  }
  bool int64(int64_t& v) {
    if (!skip()) return false;
    bool neg = false;
    if (*p == '-' || *p == '+') { neg = *p == '-'; p++; }
    if (p >= e || *p < '0' || *p > '9') return false;
    int64_t x = 0;
    while (p < e && *p >= '0' && *p <= '9') {
      x = x * 10 + (*p - '0');
      if (x > (1LL << 40)) return false;
      p++;
    }
    v = neg ? -x : x;
    return true;
  }
};

}  // namespace

bool load_calig_graph(const std::string& path, EdgeList& g, std::string& err) {
  std::string buf;
  if (!slurp(path, buf)) { err = "Fail to open graph file: " + path; return false; }
  Scan sc{buf.data(), buf.data() + buf.size()};
  g = EdgeList{};
  std::string tag;
  std::vector<int64_t> raw;
  while (sc.word(tag)) {
    if (tag == "v") {
      int64_t id, lb;
      if (!sc.int64(id) || !sc.int64(lb) || id < 0) { err = "bad vertex line in " + path; return false; }
      if (lb < 0) lb = 0;  // inputQ: a label of -1 is read as 0
      if ((uint64_t)id >= g.vlabels.size()) g.vlabels.resize((size_t)id + 1, kNotExist);
      g.vlabels[(size_t)id] = (uint32_t)lb;
    } else if (tag == "e") {
      int64_t a, b;
      if (!sc.int64(a) || !sc.int64(b)) { err = "bad edge line in " + path; return false; }
      raw.push_back(a); raw.push_back(b);
    } else {
      err = "unexpected token '" + tag + "' in " + path;
      return false;
    }
  }
  g.n = (uint32_t)g.vlabels.size();
  for (size_t i = 0; i + 1 < raw.size(); i += 2) {
    const int64_t a = raw[i], b = raw[i + 1];
    if (a < 0 || b < 0 || (uint64_t)a >= g.n || (uint64_t)b >= g.n) continue;  // inputG drops these
    g.edges.push_back((uint32_t)a); g.edges.push_back((uint32_t)b); g.edges.push_back(0);
  }
  canonicalize(g);
  g.n_elabels = std::max<uint32_t>(g.n_elabels, 1);
  return true;
}

bool load_calig_stream(const std::string& path, std::vector<Update>& s, std::string& err, uint64_t max_updates) {
  std::string buf;
  if (!slurp(path, buf)) { err = "Fail to open stream file: " + path; return false; }
  Scan sc{buf.data(), buf.data() + buf.size()};
  s.clear();
  std::string tag;
  int64_t a, b;
  while (sc.word(tag)) {
    if (!sc.int64(a) || !sc.int64(b)) { err = "bad update line in " + path; return false; }
    if (max_updates && s.size() >= max_updates) break;  // -c (inputUpdate, :1201-1212)
    Update u{};
    u.type = 'e';
    if (a < 0 && b < 0) { u.is_add = 0; u.id1 = (uint32_t)(-a - 1); u.id2 = (uint32_t)(-b - 1); }
    else if (a >= 0 && b >= 0) { u.is_add = 1; u.id1 = (uint32_t)a; u.id2 = (uint32_t)b; }
    else { err = "mixed-sign edge record in " + path; return false; }
    s.push_back(u);
  }
  return true;
}

bool save_calig_graph(const std::string& path, const EdgeList& g) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return false;
  for (uint32_t v = 0; v < g.n; v++)
    if (g.vlabels[v] != kNotExist) fprintf(f, "v %u %u\n", v, g.vlabels[v]);
  for (uint64_t i = 0; i < g.num_edges(); i++) fprintf(f, "e %u %u\n", g.edges[3 * i], g.edges[3 * i + 1]);
  return fclose(f) == 0;
}

bool save_calig_stream(const std::string& path, const std::vector<Update>& s) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return false;
  for (const Update& u : s) {
    if (u.type != 'e') continue;  // the format has no vertex records
    if (u.is_add) fprintf(f, "e %u %u\n", u.id1, u.id2);
    else fprintf(f, "e %lld %lld\n", -(long long)u.id1 - 1, -(long long)u.id2 - 1);
  }
  return fclose(f) == 0;
}

std::vector<uint8_t> calig_skipped_insertions(const EdgeList& query, const EdgeList& data,
                                              const std::vector<Update>& stream) {
  std::unordered_set<uint32_t> qlabels(query.vlabels.begin(), query.vlabels.end());
  auto valid = [&](uint32_t v) { return v < data.n && data.vlabels[v] != kNotExist && qlabels.count(data.vlabels[v]); };
  std::vector<uint8_t> entries(data.n, 0);
  for (uint64_t i = 0; i < data.num_edges(); i++) {
    const uint32_t a = data.edges[3 * i], b = data.edges[3 * i + 1];
    if (valid(a) && valid(b)) { entries[a] = 1; entries[b] = 1; }
  }
  std::unordered_set<uint64_t> skipped_edges;
  std::vector<uint8_t> skip(stream.size(), 0);
  for (size_t i = 0; i < stream.size(); i++) {
    const Update& u = stream[i];
    if (u.type != 'e' || !valid(u.id1) || !valid(u.id2) || u.id1 == u.id2) continue;
    const uint64_t k = edge_key(u.id1, u.id2);
    if (!u.is_add) { skipped_edges.erase(k); continue; }
    if (skipped_edges.count(k)) { skip[i] = 1; continue; }  // in the neighbour sets already: a duplicate
    if (!entries[u.id1]) { skip[i] = 1; skipped_edges.insert(k); continue; }
    entries[u.id2] = 1;
  }
  return skip;
}

}  // namespace csm
