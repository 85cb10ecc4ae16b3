#include "graph_io.h"

#include <algorithm>
#include <cstdio>
#include <cstring>

namespace csm {
namespace {

bool read_file(const std::string& path, std::string& buf) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  buf.resize(sz > 0 ? (size_t)sz : 0);
  size_t got = sz > 0 ? fread(&buf[0], 1, (size_t)sz, f) : 0;
  fclose(f);
  return got == buf.size();
}

struct Tok {
  const char* p;
  const char* e;
  bool word(const char*& s, size_t& n) {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
    if (p >= e) return false;
    s = p;
    while (p < e && !(*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
    n = (size_t)(p - s);
    return true;
  }
  bool u32(uint32_t& v) {
    const char* s; size_t n;
    if (!word(s, n)) return false;
    uint64_t x = 0;
    for (size_t i = 0; i < n; i++) {
      if (s[i] < '0' || s[i] > '9') return false;
      x = x * 10 + (uint64_t)(s[i] - '0');
      if (x > 0xffffffffULL) return false;
    }
    v = (uint32_t)x;
    return n > 0;
  }
};

bool has_magic(const std::string& path, const char* magic) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  char m[4] = {0, 0, 0, 0};
  size_t got = fread(m, 1, 4, f);
  fclose(f);
  return got == 4 && memcmp(m, magic, 4) == 0;
}

}  // namespace

void canonicalize(EdgeList& g) {
  // sort (undirected key, position) pairs: the first occurrence of each edge
  // keeps its label; 16 bytes per edge instead of a hash set's nodes
  struct KI { uint64_t key; uint64_t idx; };
  const uint64_t m = g.num_edges();
  std::vector<KI> ki;
  ki.reserve(m);
  for (uint64_t i = 0; i < m; i++) {
    const uint32_t a = g.edges[3 * i], b = g.edges[3 * i + 1];
    if (a == b) continue;
    ki.push_back(KI{((uint64_t)std::min(a, b) << 32) | std::max(a, b), i});
  }
  std::sort(ki.begin(), ki.end(), [](const KI& x, const KI& y) { return x.key != y.key ? x.key < y.key : x.idx < y.idx; });
  std::vector<uint64_t> keep;
  keep.reserve(ki.size());
  for (size_t j = 0; j < ki.size(); j++)
    if (j == 0 || ki[j].key != ki[j - 1].key) keep.push_back(ki[j].idx);
  std::vector<KI>().swap(ki);
  std::sort(keep.begin(), keep.end());  // file order
  std::vector<uint32_t> out;
  out.reserve(3 * keep.size());
  uint32_t max_el = 0;
  for (uint64_t i : keep) {
    const uint32_t l = g.edges[3 * i + 2];
    out.push_back(g.edges[3 * i]); out.push_back(g.edges[3 * i + 1]); out.push_back(l);
    max_el = std::max(max_el, l + 1);
  }
  g.edges.swap(out);
  uint32_t max_vl = 0;
  for (uint32_t l : g.vlabels) if (l != kNotExist) max_vl = std::max(max_vl, l + 1);
  g.n_vlabels = std::max(g.n_vlabels, max_vl);
  g.n_elabels = std::max(g.n_elabels, max_el);
}

bool load_graph_text(const std::string& path, EdgeList& g, std::string& err) {
  std::string buf;
  if (!read_file(path, buf)) { err = "Failed to open: " + path; return false; }
  Tok t{buf.data(), buf.data() + buf.size()};
  g = EdgeList{};
  const char* s; size_t n;
  while (t.word(s, n)) {
    if (n >= 1 && s[0] == 't') {  // "t # <id>": skip two tokens
      const char* s2; size_t n2;
      if (!t.word(s2, n2) || !t.word(s2, n2)) break;
      continue;
    }
    if (n == 1 && s[0] == 'v') {
      uint32_t id, l;
      if (!t.u32(id) || !t.u32(l)) { err = "bad vertex line in " + path; return false; }
      if (id >= g.vlabels.size()) g.vlabels.resize((size_t)id + 1, kNotExist);
      if (g.vlabels[id] == kNotExist) g.vlabels[id] = l;
      continue;
    }
    uint32_t a, b, l;
    if (!t.u32(a) || !t.u32(b) || !t.u32(l)) { err = "bad edge line in " + path; return false; }
    g.edges.push_back(a); g.edges.push_back(b); g.edges.push_back(l);
  }
  g.n = (uint32_t)g.vlabels.size();
  for (uint64_t i = 0; i < g.num_edges(); i++) {
    if (g.edges[3 * i] >= g.n || g.edges[3 * i + 1] >= g.n) {
      err = "edge endpoint without a vertex line in " + path;
      return false;
    }
  }
  canonicalize(g);
  return true;
}

bool load_stream_text(const std::string& path, std::vector<Update>& s, std::string& err) {
  std::string buf;
  if (!read_file(path, buf)) { err = "Failed to open: " + path; return false; }
  Tok t{buf.data(), buf.data() + buf.size()};
  s.clear();
  const char* w; size_t n;
  while (t.word(w, n)) {
    Update u{};
    bool is_v = (n == 1 && w[0] == 'v') || (n == 2 && w[0] == '-' && w[1] == 'v');
    if (is_v) {
      u.type = 'v'; u.is_add = (n == 1);
      if (!t.u32(u.id1) || !t.u32(u.label)) { err = "bad vertex update in " + path; return false; }
    } else {
      u.type = 'e'; u.is_add = (n == 1 && w[0] == 'e');
      if (!t.u32(u.id1) || !t.u32(u.id2) || !t.u32(u.label)) { err = "bad edge update in " + path; return false; }
    }
    s.push_back(u);
  }
  return true;
}

bool load_graph_binary(const std::string& path, EdgeList& g, std::string& err) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) { err = "Failed to open: " + path; return false; }
  char magic[4]; uint32_t ver = 0, n = 0, nvl = 0, nel = 0; uint64_t m = 0;
  bool ok = fread(magic, 1, 4, f) == 4 && memcmp(magic, "CSMG", 4) == 0 &&
            fread(&ver, 4, 1, f) == 1 && fread(&n, 4, 1, f) == 1 && fread(&m, 8, 1, f) == 1 &&
            fread(&nvl, 4, 1, f) == 1 && fread(&nel, 4, 1, f) == 1;
  if (ok) {
    g = EdgeList{};
    g.n = n; g.n_vlabels = nvl; g.n_elabels = nel;
    g.vlabels.resize(n);
    g.edges.resize(3 * m);
    ok = fread(g.vlabels.data(), 4, n, f) == n && fread(g.edges.data(), 4, 3 * m, f) == 3 * m;
  }
  fclose(f);
  if (!ok) { err = "bad binary graph " + path; return false; }
  for (uint64_t i = 0; i < 3 * m; i += 3)
    if (g.edges[i] >= n || g.edges[i + 1] >= n) { err = "edge endpoint out of range in " + path; return false; }
  return true;
}

bool load_stream_binary(const std::string& path, std::vector<Update>& s, std::string& err) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) { err = "Failed to open: " + path; return false; }
  char magic[4]; uint32_t ver = 0; uint64_t n = 0;
  bool ok = fread(magic, 1, 4, f) == 4 && memcmp(magic, "CSMU", 4) == 0 &&
            fread(&ver, 4, 1, f) == 1 && fread(&n, 8, 1, f) == 1;
  std::vector<uint32_t> rec;
  if (ok) { rec.resize(4 * n); ok = fread(rec.data(), 4, 4 * n, f) == 4 * n; }
  fclose(f);
  if (!ok) { err = "bad binary stream " + path; return false; }
  s.resize(n);
  for (uint64_t i = 0; i < n; i++) {
    Update u{};
    u.type = (uint8_t)(rec[4 * i] & 0xff);
    u.is_add = (uint8_t)((rec[4 * i] >> 8) & 0xff);
    u.id1 = rec[4 * i + 1]; u.id2 = rec[4 * i + 2]; u.label = rec[4 * i + 3];
    s[i] = u;
  }
  return true;
}

bool load_graph_any(const std::string& path, EdgeList& g, std::string& err) {
  return has_magic(path, "CSMG") ? load_graph_binary(path, g, err) : load_graph_text(path, g, err);
}
bool load_stream_any(const std::string& path, std::vector<Update>& s, std::string& err) {
  return has_magic(path, "CSMU") ? load_stream_binary(path, s, err) : load_stream_text(path, s, err);
}

bool save_graph_text(const std::string& path, const EdgeList& g) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return false;
  std::vector<char> buf(1 << 22);
  setvbuf(f, buf.data(), _IOFBF, buf.size());
  for (uint32_t v = 0; v < g.n; v++)
    if (g.vlabels[v] != kNotExist) fprintf(f, "v %u %u\n", v, g.vlabels[v]);
  for (uint64_t i = 0; i < g.num_edges(); i++)
    fprintf(f, "e %u %u %u\n", g.edges[3 * i], g.edges[3 * i + 1], g.edges[3 * i + 2]);
  return fclose(f) == 0;
}

bool save_stream_text(const std::string& path, const std::vector<Update>& s) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return false;
  for (const Update& u : s) {
    if (u.type == 'v') fprintf(f, "%s %u %u\n", u.is_add ? "v" : "-v", u.id1, u.label);
    else fprintf(f, "%s %u %u %u\n", u.is_add ? "e" : "-e", u.id1, u.id2, u.label);
  }
  return fclose(f) == 0;
}

bool save_graph_binary(const std::string& path, const EdgeList& g) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  uint32_t ver = 1; uint64_t m = g.num_edges();
  bool ok = fwrite("CSMG", 1, 4, f) == 4 && fwrite(&ver, 4, 1, f) == 1 && fwrite(&g.n, 4, 1, f) == 1 &&
            fwrite(&m, 8, 1, f) == 1 && fwrite(&g.n_vlabels, 4, 1, f) == 1 &&
            fwrite(&g.n_elabels, 4, 1, f) == 1 &&
            fwrite(g.vlabels.data(), 4, g.n, f) == g.n &&
            fwrite(g.edges.data(), 4, 3 * m, f) == 3 * m;
  return (fclose(f) == 0) && ok;
}

bool save_stream_binary(const std::string& path, const std::vector<Update>& s) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  uint32_t ver = 1; uint64_t n = s.size();
  std::vector<uint32_t> rec(4 * n);
  for (uint64_t i = 0; i < n; i++) {
    rec[4 * i] = (uint32_t)s[i].type | ((uint32_t)s[i].is_add << 8);
    rec[4 * i + 1] = s[i].id1; rec[4 * i + 2] = s[i].id2; rec[4 * i + 3] = s[i].label;
  }
  bool ok = fwrite("CSMU", 1, 4, f) == 4 && fwrite(&ver, 4, 1, f) == 1 && fwrite(&n, 8, 1, f) == 1 &&
            fwrite(rec.data(), 4, 4 * n, f) == 4 * n;
  return (fclose(f) == 0) && ok;
}

}  // namespace csm
