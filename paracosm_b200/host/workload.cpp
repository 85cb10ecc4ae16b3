#include "workload.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>
#include <parallel/algorithm>
#include <random>

namespace csm {
namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
inline double unit(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

struct KeyIdx {
  uint64_t key;
  uint64_t idx;
};

// Unique undirected RMAT edges, in order of first appearance in the seeded
// sample sequence.  Sample i belongs to chunk i / kChunk, whose generator is
// seeded from (seed, chunk), so the result does not depend on thread count.
std::vector<uint64_t> rmat_edges(const WorkloadSpec& s, uint64_t target) {
  const uint64_t kChunk = 1 << 16;
  const uint32_t L = s.log2_n;
  const double a = s.rmat_a, ab = s.rmat_a + s.rmat_b, abc = s.rmat_a + s.rmat_b + s.rmat_c;
  std::vector<KeyIdx> all;
  uint64_t next_chunk = 0;
  uint64_t want = (uint64_t)((double)target * 1.25) + kChunk;
  std::vector<uint64_t> uniq;
  for (int round = 0; round < 64; round++) {
    uint64_t n_chunks = (want + kChunk - 1) / kChunk;
    size_t base = all.size();
    all.resize(base + n_chunks * kChunk);
#pragma omp parallel for schedule(dynamic, 4)
    for (uint64_t c = 0; c < n_chunks; c++) {
      uint64_t chunk = next_chunk + c;
      std::mt19937_64 rng(splitmix64(s.seed * 0x100000001B3ULL + chunk));
      for (uint64_t j = 0; j < kChunk; j++) {
        uint64_t u = 0, v = 0;
        for (uint32_t lvl = 0; lvl < L; lvl++) {
          double r = unit(rng());
          uint64_t bu = 0, bv = 0;
          if (r < a) {} else if (r < ab) { bv = 1; } else if (r < abc) { bu = 1; } else { bu = 1; bv = 1; }
          u = (u << 1) | bu; v = (v << 1) | bv;
        }
        uint64_t idx = chunk * kChunk + j;
        uint64_t key = (u == v) ? ~0ULL : ((std::min(u, v) << 32) | std::max(u, v));
        all[base + c * kChunk + j] = KeyIdx{key, idx};
      }
    }
    next_chunk += n_chunks;
    // unique by key keeping the smallest sample index
    std::vector<KeyIdx> tmp(all);
    __gnu_parallel::sort(tmp.begin(), tmp.end(), [](const KeyIdx& x, const KeyIdx& y) {
      return x.key < y.key || (x.key == y.key && x.idx < y.idx);
    });
    std::vector<KeyIdx> u;
    u.reserve(tmp.size());
    for (size_t i = 0; i < tmp.size(); i++) {
      if (tmp[i].key == ~0ULL) break;
      if (i == 0 || tmp[i].key != tmp[i - 1].key) u.push_back(tmp[i]);
    }
    tmp.clear(); tmp.shrink_to_fit();
    if (u.size() >= target) {
      __gnu_parallel::sort(u.begin(), u.end(), [](const KeyIdx& x, const KeyIdx& y) { return x.idx < y.idx; });
      uniq.resize(target);
      for (uint64_t i = 0; i < target; i++) uniq[i] = u[i].key;
      return uniq;
    }
    // grow by the observed yield of unique edges per sample
    double yield = (double)u.size() / (double)all.size();
    double need = (double)(target - u.size()) / std::max(yield * 0.5, 1e-3);
    want = (uint64_t)need + kChunk;
  }
  return uniq;  // empty: could not reach the target
}

// Zipf(s) (or uniform if s == 0) cumulative table over k labels.
std::vector<double> label_cdf(uint32_t k, double s) {
  std::vector<double> w(k);
  for (uint32_t i = 0; i < k; i++) w[i] = (s == 0.0) ? 1.0 : 1.0 / std::pow((double)(i + 1), s);
  double tot = std::accumulate(w.begin(), w.end(), 0.0);
  std::vector<double> cdf(k);
  double acc = 0;
  for (uint32_t i = 0; i < k; i++) { acc += w[i] / tot; cdf[i] = acc; }
  cdf[k - 1] = 1.0;
  return cdf;
}

struct Csr {
  std::vector<uint64_t> off;
  std::vector<uint32_t> nbr, lab;
  uint32_t deg(uint32_t v) const { return (uint32_t)(off[v + 1] - off[v]); }
  // label of edge (a,b) or kNotExist
  uint32_t edge_label(uint32_t a, uint32_t b) const {
    if (deg(a) > deg(b)) std::swap(a, b);
    auto beg = nbr.begin() + (long)off[a], end = nbr.begin() + (long)off[a + 1];
    auto it = std::lower_bound(beg, end, b);
    if (it == end || *it != b) return kNotExist;
    return lab[(size_t)(it - nbr.begin())];
  }
};

Csr build_csr(const EdgeList& g) {
  Csr c;
  c.off.assign((size_t)g.n + 1, 0);
  uint64_t m = g.num_edges();
  for (uint64_t i = 0; i < m; i++) { c.off[g.edges[3 * i] + 1]++; c.off[g.edges[3 * i + 1] + 1]++; }
  for (uint32_t v = 0; v < g.n; v++) c.off[v + 1] += c.off[v];
  std::vector<uint64_t> pos(c.off.begin(), c.off.end() - 1);
  c.nbr.resize(2 * m); c.lab.resize(2 * m);
  for (uint64_t i = 0; i < m; i++) {
    uint32_t a = g.edges[3 * i], b = g.edges[3 * i + 1], l = g.edges[3 * i + 2];
    c.nbr[pos[a]] = b; c.lab[pos[a]++] = l;
    c.nbr[pos[b]] = a; c.lab[pos[b]++] = l;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (uint32_t v = 0; v < g.n; v++) {
    uint64_t b = c.off[v], e = c.off[v + 1];
    std::vector<std::pair<uint32_t, uint32_t>> t;
    t.reserve(e - b);
    for (uint64_t k = b; k < e; k++) t.emplace_back(c.nbr[k], c.lab[k]);
    std::sort(t.begin(), t.end());
    for (uint64_t k = b; k < e; k++) { c.nbr[k] = t[k - b].first; c.lab[k] = t[k - b].second; }
  }
  return c;
}

bool sample_query(const Csr& g, const EdgeList& el, const QuerySpec& qs, std::mt19937_64& rng,
                  Query& q, std::string& err) {
  const uint32_t k = qs.size;
  if (k < 2) { err = "query size must be >= 2"; return false; }
  std::vector<uint32_t> nonzero;
  for (uint32_t v = 0; v < el.n; v++) if (g.deg(v) > 0) nonzero.push_back(v);
  if (nonzero.empty()) { err = "data graph has no edges"; return false; }
  for (int attempt = 0; attempt < 20000; attempt++) {
    std::vector<uint32_t> sample;
    uint32_t cur = nonzero[rng() % nonzero.size()];
    sample.push_back(cur);
    for (uint64_t step = 0; step < 64ULL * k && sample.size() < k; step++) {
      uint32_t d = g.deg(cur);
      cur = g.nbr[g.off[cur] + rng() % d];
      if (std::find(sample.begin(), sample.end(), cur) == sample.end()) sample.push_back(cur);
    }
    if (sample.size() < k) continue;
    // induced edges, (i < j) order
    std::vector<uint32_t> ind;
    for (uint32_t i = 0; i < k; i++)
      for (uint32_t j = i + 1; j < k; j++) {
        uint32_t l = g.edge_label(sample[i], sample[j]);
        if (l != kNotExist) { ind.push_back(i); ind.push_back(j); ind.push_back(l); }
      }
    std::vector<uint32_t> edges;
    if (qs.dense) {
      double avg = 2.0 * (double)(ind.size() / 3) / (double)k;
      if (avg < qs.min_avg_degree) continue;
      edges = ind;
    } else {
      size_t ne = ind.size() / 3;
      std::vector<size_t> order(ne);
      std::iota(order.begin(), order.end(), 0);
      std::shuffle(order.begin(), order.end(), rng);
      std::vector<uint32_t> parent(k);
      std::iota(parent.begin(), parent.end(), 0);
      auto find = [&](uint32_t x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
      std::vector<char> used(ne, 0);
      for (size_t t : order) {
        uint32_t ra = find(ind[3 * t]), rb = find(ind[3 * t + 1]);
        if (ra == rb) continue;
        parent[ra] = rb; used[t] = 1;
      }
      uint32_t extra = 0;
      for (size_t t : order) {
        if (used[t] || extra >= qs.extra_edges) continue;
        used[t] = 1; extra++;
      }
      for (size_t t = 0; t < ne; t++)
        if (used[t]) { edges.push_back(ind[3 * t]); edges.push_back(ind[3 * t + 1]); edges.push_back(ind[3 * t + 2]); }
    }
    q.n = k;
    q.sample = sample;
    q.vlabels.resize(k);
    for (uint32_t i = 0; i < k; i++) q.vlabels[i] = el.vlabels[sample[i]];
    q.edges = edges;
    return true;
  }
  err = "could not sample a query of size " + std::to_string(k) + " meeting its density bound";
  return false;
}

}  // namespace

bool preset(const std::string& name, WorkloadSpec& s) {
  s = WorkloadSpec{};
  s.name = name;
  if (name == "c1") {
    s.seed = 1; s.log2_n = 14; s.avg_degree = 8; s.n_vlabels = 4; s.vlabel_zipf = 0; s.n_elabels = 1;
    s.queries = {QuerySpec{6, true, 0, 0.0}};
    s.n_updates = 2000; s.insert_fraction = 1.0; s.holdout_fraction = 0.10;
  } else if (name == "c2") {
    s.seed = 2; s.log2_n = 19; s.avg_degree = 16; s.n_vlabels = 8; s.vlabel_zipf = 1.0; s.n_elabels = 2;
    s.queries = {QuerySpec{8, false, 2, 0.0}, QuerySpec{12, false, 2, 0.0}};
    s.n_updates = 100000; s.insert_fraction = 0.9;
  } else if (name == "c3" || name == "c4") {
    s.seed = 3; s.log2_n = 22; s.avg_degree = 28; s.n_vlabels = 16; s.vlabel_zipf = 1.2; s.n_elabels = 4;
    if (name == "c3") {
      s.queries = {QuerySpec{16, true, 0, 4.0}};
      s.n_updates = 1000000; s.insert_fraction = 0.8;
    } else {
      std::mt19937_64 r(44);
      s.queries.clear();
      for (int i = 0; i < 64; i++) {
        uint32_t sz = 4 + (uint32_t)(r() % 29);
        bool dense = (i % 2) == 1;
        s.queries.push_back(QuerySpec{sz, dense, dense ? 0u : 2u, 0.0});
      }
      s.n_updates = 200000; s.insert_fraction = 0.85;
    }
  } else if (name == "c5") {
    s.seed = 5; s.log2_n = 24; s.avg_degree = 32; s.n_vlabels = 32; s.vlabel_zipf = 1.0; s.n_elabels = 4;
    s.queries = {QuerySpec{24, false, 2, 0.0}, QuerySpec{24, true, 0, 0.0},
                 QuerySpec{32, false, 2, 0.0}, QuerySpec{32, true, 0, 0.0}};
    s.n_updates = 500000; s.insert_fraction = 0.9;
  } else {
    return false;
  }
  return true;
}

bool generate(const WorkloadSpec& s, Workload& w, std::string& err) {
  w = Workload{};
  w.spec = s;
  if (s.log2_n < 2 || s.log2_n > 30) { err = "log2_n out of range"; return false; }
  const uint32_t n = 1u << s.log2_n;
  const uint64_t E = (uint64_t)std::llround((double)n * s.avg_degree / 2.0);
  std::vector<uint64_t> keys = rmat_edges(s, E);
  if (keys.size() != E) { err = "RMAT could not reach the requested edge count"; return false; }
  w.total_edges = E;

  // seeded vertex relabelling so that hubs are not clustered at small ids
  std::vector<uint32_t> perm(n);
  std::iota(perm.begin(), perm.end(), 0u);
  { std::mt19937_64 r(splitmix64(s.seed ^ 0x5045524DULL)); std::shuffle(perm.begin(), perm.end(), r); }

  EdgeList all;
  all.n = n; all.n_vlabels = s.n_vlabels; all.n_elabels = s.n_elabels;
  all.vlabels.resize(n);
  std::vector<double> cdf = label_cdf(s.n_vlabels, s.vlabel_zipf);
  for (uint32_t v = 0; v < n; v++) {
    double r = unit(splitmix64(splitmix64(s.seed ^ 0x564C4142ULL) ^ (uint64_t)v));
    all.vlabels[v] = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), r) - cdf.begin());
    if (all.vlabels[v] >= s.n_vlabels) all.vlabels[v] = s.n_vlabels - 1;
  }
  all.edges.resize(3 * E);
  const uint64_t el_seed = splitmix64(s.seed ^ 0x454C4142ULL);
  for (uint64_t i = 0; i < E; i++) {
    uint32_t a = perm[(uint32_t)(keys[i] >> 32)], b = perm[(uint32_t)(keys[i] & 0xffffffffu)];
    all.edges[3 * i] = a; all.edges[3 * i + 1] = b;
    all.edges[3 * i + 2] = (uint32_t)(splitmix64(el_seed ^ i) % s.n_elabels);
  }
  keys.clear(); keys.shrink_to_fit();

  // hold-out split by seeded shuffle
  const uint64_t n_ins = (uint64_t)std::llround((double)s.n_updates * s.insert_fraction);
  const uint64_t n_del = s.n_updates - n_ins;
  uint64_t H = s.holdout_fraction > 0 ? (uint64_t)std::llround((double)E * s.holdout_fraction) : n_ins;
  if (H < n_ins || H >= E) { err = "hold-out size does not cover the insertions"; return false; }
  std::vector<uint64_t> eorder(E);
  std::iota(eorder.begin(), eorder.end(), 0ULL);
  { std::mt19937_64 r(splitmix64(s.seed ^ 0x484F4C44ULL)); std::shuffle(eorder.begin(), eorder.end(), r); }
  std::vector<char> held(E, 0);
  for (uint64_t i = 0; i < H; i++) held[eorder[i]] = 1;

  w.initial.n = n; w.initial.n_vlabels = s.n_vlabels; w.initial.n_elabels = s.n_elabels;
  w.initial.vlabels = all.vlabels;
  w.initial.edges.reserve(3 * (E - H));
  std::vector<uint64_t> cur;  // ids (into `all`) of edges existing at the current stream position
  cur.reserve(E - H + n_ins);
  for (uint64_t i = 0; i < E; i++) {
    if (held[i]) continue;
    w.initial.edges.push_back(all.edges[3 * i]);
    w.initial.edges.push_back(all.edges[3 * i + 1]);
    w.initial.edges.push_back(all.edges[3 * i + 2]);
    cur.push_back(i);
  }

  // update stream: exact insert / delete counts in a seeded order
  std::vector<char> kinds(s.n_updates, 0);
  for (uint64_t i = 0; i < n_ins; i++) kinds[i] = 1;
  std::mt19937_64 sr(splitmix64(s.seed ^ 0x53545245ULL));
  std::shuffle(kinds.begin(), kinds.end(), sr);
  uint64_t next_ins = 0;
  w.stream.reserve(s.n_updates);
  auto take_snapshot = [&]() {
    w.snapshot.n = n; w.snapshot.n_vlabels = s.n_vlabels; w.snapshot.n_elabels = s.n_elabels;
    w.snapshot.vlabels = all.vlabels;
    std::vector<uint64_t> ids(cur);
    std::sort(ids.begin(), ids.end());
    w.snapshot.edges.resize(3 * ids.size());
    for (size_t k = 0; k < ids.size(); k++)
      for (int c = 0; c < 3; c++) w.snapshot.edges[3 * k + c] = all.edges[3 * ids[k] + c];
  };
  if (s.snapshot_at > s.n_updates) { err = "snapshot position beyond the stream"; return false; }
  for (uint64_t i = 0; i < s.n_updates; i++) {
    if (s.snapshot_at && i == s.snapshot_at) take_snapshot();
    Update u{};
    u.type = 'e';
    if (kinds[i]) {
      uint64_t id = eorder[next_ins++];
      u.is_add = 1; u.id1 = all.edges[3 * id]; u.id2 = all.edges[3 * id + 1]; u.label = all.edges[3 * id + 2];
      cur.push_back(id);
    } else {
      uint64_t j = sr() % cur.size();
      uint64_t id = cur[j];
      cur[j] = cur.back(); cur.pop_back();
      u.is_add = 0; u.id1 = all.edges[3 * id]; u.id2 = all.edges[3 * id + 1]; u.label = all.edges[3 * id + 2];
    }
    w.stream.push_back(u);
  }
  if (s.snapshot_at && s.snapshot_at == s.n_updates) take_snapshot();
  (void)n_del;

  // queries sampled from the initial graph
  Csr g = build_csr(w.initial);
  std::mt19937_64 qr(splitmix64(s.seed ^ 0x51554552ULL));
  for (const QuerySpec& qs : s.queries) {
    Query q;
    if (!sample_query(g, w.initial, qs, qr, q, err)) return false;
    w.queries.push_back(q);
  }
  return true;
}

bool save_query_text(const std::string& path, const Query& q) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return false;
  for (uint32_t i = 0; i < q.n; i++) fprintf(f, "v %u %u\n", i, q.vlabels[i]);
  for (size_t i = 0; i < q.edges.size(); i += 3) fprintf(f, "e %u %u %u\n", q.edges[i], q.edges[i + 1], q.edges[i + 2]);
  return fclose(f) == 0;
}

}  // namespace csm
