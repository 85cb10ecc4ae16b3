// CPU restatement of ParaCOSM's per-update matching semantics.
// TEST INFRASTRUCTURE ONLY (see csm_oracle.h): the checker, never the product.
#include "csm_oracle.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace {

const uint32_t NOT_EXIST = 0xffffffffu;

inline uint64_t mix64(uint64_t x) {  // MurmurHash3 fmix64 (public domain)
  x ^= x >> 33; x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33; return x;
}
inline uint64_t pair_hash(uint32_t q, uint32_t v) {
  return mix64((((uint64_t)(q + 1)) << 32) ^ (uint64_t)v ^ 0x9E3779B97F4A7C15ULL);
}

// Adjacency kept sorted by neighbour id with a parallel edge-label list
// (ParaCOSM/CSM/graph/graph.h:63-100, graph.cpp:58-116).
struct Graph {
  std::vector<uint32_t> vlabel;
  std::vector<std::vector<uint32_t>> nbr, elab;
  uint32_t n_el = 1, n_vl = 1;
  // segment sizes |S(v, a, l)| for the byte model, indexed v * n_vl * n_el + a * n_el + l
  std::vector<uint32_t> seg;
  bool track_seg = false;

  uint32_t label(uint32_t v) const { return v < vlabel.size() ? vlabel[v] : NOT_EXIST; }
  uint32_t deg(uint32_t v) const { return (uint32_t)nbr[v].size(); }
  size_t combo(uint32_t a, uint32_t l) const { return (size_t)a * n_el + l; }

  void add_vertex(uint32_t id, uint32_t l) {  // graph.cpp:23-49
    if (id >= vlabel.size()) {
      vlabel.resize((size_t)id + 1, NOT_EXIST);
      nbr.resize((size_t)id + 1);
      elab.resize((size_t)id + 1);
      if (track_seg) seg.resize(((size_t)id + 1) * n_vl * n_el, 0);
      vlabel[id] = l;
    } else if (vlabel[id] == NOT_EXIST) {
      vlabel[id] = l;
    }
  }
  void seg_adj(uint32_t v, uint32_t w, uint32_t l, int d) {
    if (!track_seg) return;
    uint32_t a = label(w);
    if (a == NOT_EXIST || a >= n_vl || l >= n_el) return;
    seg[(size_t)v * n_vl * n_el + combo(a, l)] += (uint32_t)d;
  }
  // returns false if the edge already existed (graph.cpp:63-64)
  bool add_edge(uint32_t a, uint32_t b, uint32_t l) {
    auto it = std::lower_bound(nbr[a].begin(), nbr[a].end(), b);
    if (it != nbr[a].end() && *it == b) return false;
    size_t d = (size_t)(it - nbr[a].begin());
    nbr[a].insert(it, b); elab[a].insert(elab[a].begin() + (long)d, l);
    it = std::lower_bound(nbr[b].begin(), nbr[b].end(), a);
    d = (size_t)(it - nbr[b].begin());
    nbr[b].insert(it, a); elab[b].insert(elab[b].begin() + (long)d, l);
    seg_adj(a, b, l, +1); seg_adj(b, a, l, +1);
    return true;
  }
  // returns false if the edge is missing (the reference exits, graph.cpp:98-109)
  bool remove_edge(uint32_t a, uint32_t b) {
    auto it = std::lower_bound(nbr[a].begin(), nbr[a].end(), b);
    if (it == nbr[a].end() || *it != b) return false;
    size_t d = (size_t)(it - nbr[a].begin());
    uint32_t l = elab[a][d];
    nbr[a].erase(it); elab[a].erase(elab[a].begin() + (long)d);
    it = std::lower_bound(nbr[b].begin(), nbr[b].end(), a);
    if (it == nbr[b].end() || *it != a) return false;
    d = (size_t)(it - nbr[b].begin());
    nbr[b].erase(it); elab[b].erase(elab[b].begin() + (long)d);
    seg_adj(a, b, l, -1); seg_adj(b, a, l, -1);
    return true;
  }
  // edge label or NOT_EXIST (graph.cpp:133-174)
  uint32_t edge_label(uint32_t a, uint32_t b) const {
    if (a >= nbr.size() || b >= nbr.size()) return NOT_EXIST;
    uint32_t x = deg(a) < deg(b) ? a : b, y = (x == a) ? b : a;
    auto it = std::lower_bound(nbr[x].begin(), nbr[x].end(), y);
    if (it == nbr[x].end() || *it != y) return NOT_EXIST;
    return elab[x][(size_t)(it - nbr[x].begin())];
  }
  uint32_t seg_size(uint32_t v, uint32_t a, uint32_t l) const {
    if (a >= n_vl || l >= n_el) return 0;
    return seg[(size_t)v * n_vl * n_el + combo(a, l)];
  }
};

struct QueryGraph {
  uint32_t n = 0;
  std::vector<uint32_t> vlabel;
  std::vector<std::vector<uint32_t>> nbr, elab;  // sorted by id like Graph
  uint32_t n_edges = 0;
  bool build(uint32_t nv, const uint32_t* vl, uint32_t ne, const uint32_t* e) {
    n = nv; vlabel.assign(vl, vl + nv); nbr.assign(nv, {}); elab.assign(nv, {});
    for (uint32_t i = 0; i < ne; i++) {
      uint32_t a = e[3 * i], b = e[3 * i + 1], l = e[3 * i + 2];
      if (a >= nv || b >= nv || a == b) return false;
      auto it = std::lower_bound(nbr[a].begin(), nbr[a].end(), b);
      if (it != nbr[a].end() && *it == b) continue;
      size_t d = (size_t)(it - nbr[a].begin());
      nbr[a].insert(it, b); elab[a].insert(elab[a].begin() + (long)d, l);
      it = std::lower_bound(nbr[b].begin(), nbr[b].end(), a);
      d = (size_t)(it - nbr[b].begin());
      nbr[b].insert(it, a); elab[b].insert(elab[b].begin() + (long)d, l);
      n_edges++;
    }
    return true;
  }
  uint32_t deg(uint32_t u) const { return (uint32_t)nbr[u].size(); }
  uint32_t edge_label(uint32_t a, uint32_t b) const {
    auto it = std::lower_bound(nbr[a].begin(), nbr[a].end(), b);
    if (it == nbr[a].end() || *it != b) return NOT_EXIST;
    return elab[a][(size_t)(it - nbr[a].begin())];
  }
};

// GraphFlow::GenerateMatchingOrder (graphflow.cpp:36-169): one order per query
// edge; order 0 starts at the max-degree vertex, order i > 0 starts at the
// i-th backward edge of order 0.  Each next vertex maximises the number of
// already-ordered neighbours, ties broken by larger degree, then smaller id.
void graphflow_orders(const QueryGraph& q, std::vector<std::vector<uint32_t>>& order) {
  const uint32_t n = q.n, m = q.n_edges;
  order.assign(std::max<uint32_t>(m, 1), std::vector<uint32_t>(n, 0));
  std::vector<uint32_t> offs(n, 0), csr(m + 1, 0);
  auto pick = [&](std::vector<char>& vis) {
    uint32_t best = NOT_EXIST, best_adj = 0;
    for (uint32_t j = 0; j < n; j++) {
      if (vis[j]) continue;
      uint32_t adj = 0;
      for (uint32_t o : q.nbr[j]) if (vis[o]) adj++;
      if (!adj) continue;
      if (best == NOT_EXIST || (adj == best_adj && q.deg(j) > q.deg(best)) || adj > best_adj) {
        best_adj = adj; best = j;
      }
    }
    return best;
  };
  std::vector<char> vis(n, 0);
  uint32_t maxd = 0;
  for (uint32_t i = 0; i < n; i++) if (q.deg(i) > maxd) { maxd = q.deg(i); order[0][0] = i; }
  vis[order[0][0]] = 1;
  for (uint32_t i = 1; i < n; i++) {
    uint32_t u = pick(vis);
    order[0][i] = u; vis[u] = 1;
    offs[i] = offs[i - 1];
    for (uint32_t o : q.nbr[u]) if (vis[o]) csr[offs[i]++] = o;
  }
  for (uint32_t i = 1; i < m; i++) {
    std::vector<char> v2(n, 0);
    uint32_t p = (uint32_t)(std::lower_bound(offs.begin(), offs.end(), i + 1) - offs.begin());
    order[i][0] = order[0][p];
    order[i][1] = csr[i];
    v2[order[i][0]] = 1; v2[order[i][1]] = 1;
    for (uint32_t j = 2; j < n; j++) {
      uint32_t u = pick(v2);
      order[i][j] = u; v2[u] = 1;
    }
  }
}

struct Searcher {
  const QueryGraph& q;
  Graph& g;
  const std::vector<std::vector<uint32_t>>& order;
  bool homo, want_hash;
  uint64_t cap;  // 0 = none
  std::vector<uint32_t> m;
  std::vector<char> visited;
  uint64_t count = 0, hash = 0, bytes = 0;
  bool capped = false;

  Searcher(const QueryGraph& q_, Graph& g_, const std::vector<std::vector<uint32_t>>& o, bool h, bool wh, uint64_t c)
      : q(q_), g(g_), order(o), homo(h), want_hash(wh), cap(c) {}

  // GraphFlow::FindMatches (graphflow.cpp:181-265)
  void find(uint32_t oi, uint32_t depth, uint64_t hsum) {
    const uint32_t u = order[oi][depth];
    const auto& qn = q.nbr[u];
    const auto& ql = q.elab[u];
    uint32_t u_min = NOT_EXIST, u_min_label = NOT_EXIST, u_min_size = 0xffffffffu;
    uint64_t node_bytes = 0;
    for (size_t i = 0; i < qn.size(); i++) {
      if (m[qn[i]] == NOT_EXIST) continue;
      uint32_t sz = g.deg(m[qn[i]]);
      if (sz < u_min_size) { u_min_size = sz; u_min = qn[i]; u_min_label = ql[i]; }
      node_bytes += 4ULL * g.seg_size(m[qn[i]], q.vlabel[u], ql[i]);
    }
    bytes += node_bytes;
    const uint32_t vm = m[u_min];
    const auto& dn = g.nbr[vm];
    const auto& dl = g.elab[vm];
    for (size_t i = 0; i < dn.size(); i++) {
      const uint32_t v = dn[i];
      if (g.label(v) != q.vlabel[u] || dl[i] != u_min_label) continue;
      bool ok = true;
      for (size_t j = 0; j < qn.size() && ok; j++) {
        const uint32_t uo = qn[j];
        if (m[uo] == NOT_EXIST || uo == u_min) continue;
        const auto& on = g.nbr[m[uo]];
        auto it = std::lower_bound(on.begin(), on.end(), v);
        if (it == on.end() || *it != v || g.elab[m[uo]][(size_t)(it - on.begin())] != ql[j]) ok = false;
      }
      if (!ok) continue;
      if (!homo && visited[v]) continue;
      const uint64_t h2 = want_hash ? hsum + pair_hash(u, v) : 0;
      m[u] = v; visited[v] = 1;
      if (depth == q.n - 1) {
        count++;
        if (want_hash) hash += mix64(h2);
      } else {
        find(oi, depth + 1, h2);
      }
      visited[v] = 0; m[u] = NOT_EXIST;
      if (cap && count >= cap) { capped = true; return; }
    }
  }

  // seeds of GraphFlow::AddEdge (graphflow.cpp:305-352); for deletions the
  // same embedding set is seeded with the existing edge's label
  // (graphflow.cpp:361-411).
  void run_update(uint32_t v1, uint32_t v2, uint32_t label) {
    count = hash = 0; capped = false;
    const uint32_t l1 = g.label(v1), l2 = g.label(v2);
    for (uint32_t i = 0; i < q.n_edges && !capped; i++) {
      const uint32_t u1 = order[i][0], u2 = order[i][1];
      const uint32_t el = q.edge_label(u1, u2);
      for (int orient = 0; orient < 2 && !capped; orient++) {
        const uint32_t a = orient ? v2 : v1, b = orient ? v1 : v2;
        const uint32_t la = orient ? l2 : l1, lb = orient ? l1 : l2;
        if (!(q.vlabel[u1] == la && q.vlabel[u2] == lb && el == label)) continue;
        if (q.n == 2) {
          count++;
          if (want_hash) hash += mix64(pair_hash(u1, a) + pair_hash(u2, b));
          if (cap && count >= cap) capped = true;
          continue;
        }
        m[u1] = a; m[u2] = b; visited[a] = 1; visited[b] = 1;
        find(i, 2, want_hash ? pair_hash(u1, a) + pair_hash(u2, b) : 0);
        visited[a] = 0; visited[b] = 0; m[u1] = NOT_EXIST; m[u2] = NOT_EXIST;
      }
    }
    if (capped) { count = cap; hash = 0; }
  }
};

}  // namespace

extern "C" int oracle_graphflow_orders(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe,
                                       const uint32_t* q_edges, uint32_t* out) {
  QueryGraph q;
  if (!q.build(n_qv, q_vlabels, n_qe, q_edges)) return -1;
  std::vector<std::vector<uint32_t>> order;
  graphflow_orders(q, order);
  for (uint32_t i = 0; i < q.n_edges; i++)
    for (uint32_t j = 0; j < n_qv; j++) out[(size_t)i * n_qv + j] = order[i][j];
  return (int)q.n_edges;
}

extern "C" int oracle_run(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                          uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
                          uint64_t n_up, const oracle_update* ups, uint64_t max_results, int homo,
                          int want_hash, oracle_result* out) {
  QueryGraph q;
  if (n_qv < 2 || !q.build(n_qv, q_vlabels, n_qe, q_edges) || q.n_edges == 0) return -1;
  Graph g;
  uint32_t max_vl = 0, max_el = 0;
  for (uint32_t v = 0; v < n_v; v++) if (vlabels[v] != NOT_EXIST) max_vl = std::max(max_vl, vlabels[v] + 1);
  for (uint32_t u = 0; u < n_qv; u++) max_vl = std::max(max_vl, q_vlabels[u] + 1);
  for (uint64_t i = 0; i < n_e; i++) max_el = std::max(max_el, edges[3 * i + 2] + 1);
  for (uint32_t i = 0; i < n_qe; i++) max_el = std::max(max_el, q_edges[3 * i + 2] + 1);
  for (uint64_t i = 0; i < n_up; i++) {
    if (ups[i].type == 'v') max_vl = std::max(max_vl, ups[i].label + 1);
    else max_el = std::max(max_el, ups[i].label + 1);
  }
  g.n_vl = std::max<uint32_t>(max_vl, 1); g.n_el = std::max<uint32_t>(max_el, 1);
  g.track_seg = true;
  for (uint32_t v = 0; v < n_v; v++) g.add_vertex(v, vlabels[v]);
  if (g.vlabel.size() < n_v) { g.vlabel.resize(n_v, NOT_EXIST); g.nbr.resize(n_v); g.elab.resize(n_v); g.seg.resize((size_t)n_v * g.n_vl * g.n_el, 0); }
  // sorted (min, max) insertion keeps every insert an append
  std::vector<uint64_t> idx(n_e);
  for (uint64_t i = 0; i < n_e; i++) idx[i] = i;
  auto key = [&](uint64_t i) {
    uint32_t a = edges[3 * i], b = edges[3 * i + 1];
    return ((uint64_t)std::min(a, b) << 32) | std::max(a, b);
  };
  std::stable_sort(idx.begin(), idx.end(), [&](uint64_t x, uint64_t y) { return key(x) < key(y); });
  for (uint64_t i : idx) {
    uint32_t a = edges[3 * i], b = edges[3 * i + 1];
    if (a >= n_v || b >= n_v || a == b) continue;
    g.add_edge(a, b, edges[3 * i + 2]);
  }
  std::vector<std::vector<uint32_t>> order;
  graphflow_orders(q, order);
  Searcher s(q, g, order, homo != 0, want_hash != 0, max_results);
  s.m.assign(n_qv, NOT_EXIST);
  s.visited.assign(g.vlabel.size(), 0);

  for (uint64_t i = 0; i < n_up; i++) {
    const oracle_update& u = ups[i];
    oracle_result r{};
    if (u.type == 'v') {
      if (u.is_add) {  // graphflow.cpp:418-423
        g.add_vertex(u.id1, u.label);
        if (s.visited.size() < g.vlabel.size()) s.visited.resize(g.vlabel.size(), 0);
      } else if (u.id1 < g.vlabel.size()) {
        // graph.cpp:51-56 clears the vertex; its incident edges are dropped on both sides here
        std::vector<uint32_t> ns = g.nbr[u.id1];
        for (uint32_t w : ns) g.remove_edge(u.id1, w);
        g.vlabel[u.id1] = NOT_EXIST;
      } else {
        r.status = ORACLE_INVALID;
      }
      r.safe = 1;
      out[i] = r;
      continue;
    }
    const uint32_t v1 = u.id1, v2 = u.id2;
    if (v1 >= g.vlabel.size() || v2 >= g.vlabel.size() || v1 == v2) {
      r.status = ORACLE_INVALID; r.safe = 1; out[i] = r; continue;
    }
    // label-triple safe test (parallel_graphflow.cpp:1990-2016)
    uint32_t lbl = u.is_add ? u.label : g.edge_label(v1, v2);
    bool any = false;
    for (uint32_t a = 0; a < q.n && !any; a++)
      for (size_t k = 0; k < q.nbr[a].size(); k++) {
        uint32_t b = q.nbr[a][k];
        if (q.vlabel[a] == g.label(v1) && q.vlabel[b] == g.label(v2) && q.elab[a][k] == lbl) { any = true; break; }
      }
    r.safe = any ? 0 : 1;
    s.bytes = 0;
    if (u.is_add) {
      bool added = g.add_edge(v1, v2, u.label);
      if (added) s.bytes += 16;
      s.run_update(v1, v2, u.label);
      r.pos = s.count;
    } else {
      if (lbl == NOT_EXIST) { r.status = ORACLE_INVALID; out[i] = r; continue; }
      s.run_update(v1, v2, lbl);
      r.neg = s.count;
      g.remove_edge(v1, v2);
      s.bytes += 16;
    }
    r.hash = s.hash;
    r.bytes = s.bytes;
    if (s.capped) r.status = ORACLE_CAPPED;
    out[i] = r;
  }
  return 0;
}

extern "C" int oracle_brute_count(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                                  uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
                                  uint32_t v1, uint32_t v2, int homo, uint64_t* count, uint64_t* hash) {
  // Appendix-style definition: every map f with L(f(u)) = L(u), every query
  // edge present with its label, injective unless homo, and some query edge
  // mapped onto {v1, v2}.  Exhaustive over n_v^n_qv with edge-by-edge pruning.
  QueryGraph q;
  if (!q.build(n_qv, q_vlabels, n_qe, q_edges)) return -1;
  Graph g;
  g.n_vl = 1; g.n_el = 1;
  for (uint32_t v = 0; v < n_v; v++) g.add_vertex(v, vlabels[v]);
  for (uint64_t i = 0; i < n_e; i++) {
    uint32_t a = edges[3 * i], b = edges[3 * i + 1];
    if (a < n_v && b < n_v && a != b) g.add_edge(a, b, edges[3 * i + 2]);
  }
  std::vector<uint32_t> f(n_qv, NOT_EXIST);
  uint64_t c = 0, h = 0;
  std::vector<uint32_t> cand;
  // recursive lambda over query vertices in id order
  struct Rec {
    const QueryGraph& q; const Graph& g; std::vector<uint32_t>& f; bool homo;
    uint32_t v1, v2; uint64_t& c; uint64_t& h;
    void go(uint32_t u) {
      if (u == q.n) {
        // one count per query edge mapped onto {v1, v2}: the seeds of
        // graphflow.cpp:305-352 enumerate each (map, anchor edge) pair once,
        // which is one per map unless homomorphism lets several edges map there
        uint64_t anchors = 0;
        for (uint32_t a = 0; a < q.n; a++)
          for (uint32_t b : q.nbr[a])
            if (a < b && ((f[a] == v1 && f[b] == v2) || (f[a] == v2 && f[b] == v1))) anchors++;
        if (!anchors) return;
        c += anchors;
        uint64_t s = 0;
        for (uint32_t k = 0; k < q.n; k++) s += pair_hash(k, f[k]);
        h += anchors * mix64(s);
        return;
      }
      for (uint32_t v = 0; v < g.vlabel.size(); v++) {
        if (g.label(v) != q.vlabel[u]) continue;
        if (!homo) { bool used = false; for (uint32_t k = 0; k < u; k++) if (f[k] == v) { used = true; break; }
                     if (used) continue; }
        bool ok = true;
        for (size_t k = 0; k < q.nbr[u].size() && ok; k++) {
          uint32_t w = q.nbr[u][k];
          if (w >= u) continue;
          if (g.edge_label(v, f[w]) != q.elab[u][k]) ok = false;
        }
        if (!ok) continue;
        f[u] = v;
        go(u + 1);
        f[u] = NOT_EXIST;
      }
    }
  } rec{q, g, f, homo != 0, v1, v2, c, h};
  rec.go(0);
  *count = c; *hash = h;
  return 0;
}
