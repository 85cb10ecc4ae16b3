// CPU restatement of ParaCOSM's per-update matching semantics.
// TEST INFRASTRUCTURE ONLY (see csm_oracle.h): the checker, never the product.
#include "csm_oracle.h"

#include <algorithm>
#include <functional>
#include <map>
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
    if (!track_seg || a >= n_vl || l >= n_el) return 0;
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

// Independent tail of an order (the engine's counting search, not in the
// reference): the longest suffix o[s..n-1], s >= 2, with no query edge inside
// it and no vertex label more than kTailGroup times.  Every tail vertex has
// all its neighbours before s, so given a match of o[0..s-1] the tail
// vertices only interact through injectivity, which only binds vertices of
// one label: the completions are the product over label groups of each
// group's number of injective assignments.  Returns s - 1 (the last position
// matched one by one) when the tail has at least two vertices, else 0.
constexpr uint32_t kTailGroup = 3;

uint32_t independent_tail(const QueryGraph& q, const std::vector<uint32_t>& o) {
  const uint32_t n = q.n;
  if (n < 4) return 0;
  std::vector<int> pos(n);
  for (uint32_t i = 0; i < n; i++) pos[o[i]] = (int)i;
  uint32_t s = n - 1;
  while (s > 2) {
    const uint32_t u = o[s - 1];
    bool stop = false;
    for (uint32_t w : q.nbr[u]) if (pos[w] >= (int)s) stop = true;  // an edge into the tail
    uint32_t same = 0;
    for (uint32_t i = s; i < n; i++) same += q.vlabel[o[i]] == q.vlabel[u];
    if (stop || same >= kTailGroup) break;
    s--;
  }
  return n - s >= 2 ? s - 1 : 0;
}

// Number of injective assignments of a group of g members given, for each
// nonempty membership set M (bit i: the element is a candidate of member i),
// the number N[M] of elements with exactly that membership: members served by
// elements of one class M are a subset R of M, in N[M] * (N[M]-1) * ... ways.
// Without injectivity (homo) it is the product of the members' candidate
// counts.  Saturates at kSat.
uint64_t group_assignments(uint32_t g, const uint64_t* N, bool homo) {
  const uint64_t kSat = 1ULL << 58;
  auto mul = [&](uint64_t a, uint64_t b) { return (a == 0 || b == 0) ? 0 : (a > kSat / b ? kSat : std::min(kSat, a * b)); };
  const uint32_t full = (1u << g) - 1;
  if (homo) {
    uint64_t prod = 1;
    for (uint32_t i = 0; i < g; i++) {
      uint64_t c = 0;
      for (uint32_t M = 1; M <= full; M++) if (M >> i & 1) c = std::min(kSat, c + N[M]);
      prod = mul(prod, c);
    }
    return prod;
  }
  uint64_t f[1u << kTailGroup] = {1};
  for (uint32_t M = 1; M <= full; M++) {
    if (!N[M]) continue;
    uint64_t h[1u << kTailGroup] = {0};
    for (uint32_t S = 0; S <= full; S++) {
      if (!f[S]) continue;
      const uint32_t free_ = M & ~S;
      for (uint32_t R = free_;; R = (R - 1) & free_) {  // every subset R of free_, R = 0 included
        uint64_t ways = 1;
        for (uint32_t r = 0, k = (uint32_t)__builtin_popcount(R); r < k; r++) ways = mul(ways, N[M] - r);
        if (ways) h[S | R] = std::min(kSat, h[S | R] + mul(f[S], ways));
        if (R == 0) break;
      }
    }
    for (uint32_t S = 0; S <= full; S++) f[S] = h[S];
  }
  return f[full];
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
  // per order: last position matched one by one before the independent tail
  // (0: no tail counting for that order)
  std::vector<uint32_t> tail_at;

  Searcher(const QueryGraph& q_, Graph& g_, const std::vector<std::vector<uint32_t>>& o, bool h, bool wh, uint64_t c)
      : q(q_), g(g_), order(o), homo(h), want_hash(wh), cap(c) {}

  // Is data vertex v a candidate of query vertex u under the current prefix
  // (label, adjacency with the edge label to every matched neighbour,
  // injectivity against the prefix)?
  bool is_candidate(uint32_t u, uint32_t v) {
    if (g.label(v) != q.vlabel[u]) return false;
    if (!homo && visited[v]) return false;
    const auto& qn = q.nbr[u];
    const auto& ql = q.elab[u];
    for (size_t j = 0; j < qn.size(); j++) {
      const uint32_t uo = qn[j];
      if (m[uo] == NOT_EXIST) continue;
      const auto& on = g.nbr[m[uo]];
      auto it = std::lower_bound(on.begin(), on.end(), v);
      if (it == on.end() || *it != v || g.elab[m[uo]][(size_t)(it - on.begin())] != ql[j]) return false;
    }
    return true;
  }

  // Candidates of query vertex u (scanning its smallest back neighbour's
  // list); adds the node's algorithmic bytes.
  void candidates(uint32_t u, std::vector<uint32_t>& out) {
    out.clear();
    const auto& qn = q.nbr[u];
    const auto& ql = q.elab[u];
    uint32_t u_min = NOT_EXIST, u_min_size = 0xffffffffu;
    for (size_t i = 0; i < qn.size(); i++) {
      if (m[qn[i]] == NOT_EXIST) continue;
      const uint32_t sz = g.deg(m[qn[i]]);
      if (sz < u_min_size) { u_min_size = sz; u_min = qn[i]; }
      bytes += 4ULL * g.seg_size(m[qn[i]], q.vlabel[u], ql[i]);
    }
    for (uint32_t v : g.nbr[m[u_min]])
      if (is_candidate(u, v)) out.push_back(v);
  }

  // The independent tail (independent_tail) from position `first` on: label
  // groups in order of their first position, members in position order.  For
  // each group, every member's candidates are listed (adding its bytes) and
  // classified by membership in the group's other members; an element is
  // counted once, under the first member it is a candidate of.  A group is
  // only looked at while the product is nonzero.  As in the engine, a prefix
  // whose first tail position has an empty back-neighbour segment stops
  // there (the engine drops it before the tail is looked at).
  void count_tail(uint32_t oi, uint32_t first) {
    const uint64_t kSat = 1ULL << 58;
    const auto& o = order[oi];
    {
      const uint32_t u = o[first];
      bool empty = false;
      uint64_t b = 0;
      for (size_t i = 0; i < q.nbr[u].size(); i++) {
        const uint32_t sz = g.seg_size(m[q.nbr[u][i]], q.vlabel[u], q.elab[u][i]);
        b += 4ULL * sz;
        if (sz == 0) empty = true;
      }
      if (empty) { bytes += b; return; }
    }
    std::vector<char> done(q.n, 0);
    uint64_t prod = 1;
    std::vector<uint32_t> c;
    for (uint32_t d = first; d < q.n && prod; d++) {
      if (done[d]) continue;
      std::vector<uint32_t> grp;
      for (uint32_t e = d; e < q.n; e++)
        if (!done[e] && q.vlabel[o[e]] == q.vlabel[o[d]]) { grp.push_back(e); done[e] = 1; }
      uint64_t N[1u << kTailGroup] = {0};
      for (uint32_t j = 0; j < grp.size(); j++) {
        candidates(o[grp[j]], c);
        for (uint32_t x : c) {
          uint32_t M = 1u << j;
          bool seen = false;
          for (uint32_t i = 0; i < grp.size() && !seen; i++) {
            if (i == j || !is_candidate(o[grp[i]], x)) continue;
            if (i < j) seen = true; else M |= 1u << i;
          }
          if (!seen) N[M]++;
        }
      }
      const uint64_t w = group_assignments((uint32_t)grp.size(), N, homo);
      prod = w == 0 ? 0 : (prod > kSat / w ? kSat : std::min(kSat, prod * w));
    }
    count += prod;
    if (cap && count >= cap) capped = true;
  }

  // GraphFlow::FindMatches (graphflow.cpp:181-265)
  void find(uint32_t oi, uint32_t depth, uint64_t hsum) {
    if (!tail_at.empty() && tail_at[oi] && depth == tail_at[oi] + 1) { count_tail(oi, depth); return; }
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
  std::vector<uint32_t> tail_at;
  if (!want_hash)  // counting only: the tail of each order is counted, not enumerated
    for (const auto& o : order) tail_at.push_back(independent_tail(q, o));
  Searcher s(q, g, order, homo != 0, want_hash != 0, max_results);
  s.tail_at = tail_at;
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

// ---- candidate index of the TurboFlux / SymBi plugins --------------------
namespace {

// Root choice shared by both plugins (ParaCOSM/CSM/matching/SymBi/symbi.cpp:113-195,
// TurboFlux/turboflux.cpp:69-149): per query edge (u < u', in adjacency
// order) the number of directed data entries v -> v' with L(v) = L(u),
// L(v') = L(u') and the edge's label; the first least-frequent edge gives
// the candidates, the endpoint whose label is rarer in the data graph wins,
// ties go to the larger query degree (then the second endpoint).
uint32_t dag_root(const QueryGraph& q, const Graph& g, std::vector<std::vector<uint64_t>>& freq) {
  freq.assign(q.n, std::vector<uint64_t>(q.n, 0));
  uint64_t min_freq = ~0ULL;
  uint32_t mv0 = 0, mv1 = 0;
  for (uint32_t u = 0; u < q.n; u++)
    for (size_t i = 0; i < q.nbr[u].size(); i++) {
      const uint32_t uo = q.nbr[u][i], lo = q.elab[u][i];
      if (u > uo) { freq[u][uo] = freq[uo][u]; continue; }
      uint64_t f = 0;
      for (uint32_t v = 0; v < g.vlabel.size(); v++) {
        if (g.vlabel[v] == NOT_EXIST || g.vlabel[v] != q.vlabel[u]) continue;
        for (size_t j = 0; j < g.nbr[v].size(); j++)
          if (g.label(g.nbr[v][j]) == q.vlabel[uo] && g.elab[v][j] == lo) f++;
      }
      freq[u][uo] = f;
      if (f < min_freq) { min_freq = f; mv0 = u; mv1 = uo; }
    }
  uint64_t c0 = 0, c1 = 0;
  for (uint32_t v = 0; v < g.vlabel.size(); v++) {
    if (g.vlabel[v] == NOT_EXIST) continue;
    if (g.vlabel[v] == q.vlabel[mv0]) c0++;
    if (g.vlabel[v] == q.vlabel[mv1]) c1++;
  }
  if (c0 > c1) return mv1;
  if (c0 < c1) return mv0;
  return q.deg(mv0) > q.deg(mv1) ? mv0 : mv1;
}

struct Dag {
  uint32_t root = 0;
  std::vector<uint32_t> order;                 // serialized tree
  std::vector<std::vector<uint32_t>> par, chd;  // DAG parents / children with edge labels below
  std::vector<std::vector<uint32_t>> par_l, chd_l;
};

// SymBi (symbi.cpp:197-238): BFS from the root over all query edges; an edge
// points from the endpoint dequeued first to the other one.
void dag_symbi(const QueryGraph& q, uint32_t root, Dag& d) {
  d.root = root;
  d.order.clear();
  d.par.assign(q.n, {}); d.chd.assign(q.n, {}); d.par_l.assign(q.n, {}); d.chd_l.assign(q.n, {});
  std::vector<char> seen(q.n, 0), popped(q.n, 0);
  std::vector<uint32_t> fifo{root};
  seen[root] = 1;
  d.order.push_back(root);
  for (size_t h = 0; h < fifo.size(); h++) {
    const uint32_t u = fifo[h];
    popped[u] = 1;
    for (size_t i = 0; i < q.nbr[u].size(); i++) {
      const uint32_t w = q.nbr[u][i];
      if (!seen[w]) { seen[w] = 1; fifo.push_back(w); d.order.push_back(w); }
      if (!popped[w]) {
        d.chd[u].push_back(w); d.chd_l[u].push_back(q.elab[u][i]);
        d.par[w].push_back(u); d.par_l[w].push_back(q.elab[u][i]);
      }
    }
  }
}

// TurboFlux (turboflux.cpp:151-219): a spanning tree grown level by level;
// inside a level the cheapest pending edge (first of equal frequency) is
// taken and every other pending edge into the same vertex is dropped.  The
// serialized tree is the BFS order over tree children.
void dag_turboflux(const QueryGraph& q, uint32_t root, const std::vector<std::vector<uint64_t>>& freq, Dag& d) {
  d.root = root;
  d.par.assign(q.n, {}); d.chd.assign(q.n, {}); d.par_l.assign(q.n, {}); d.chd_l.assign(q.n, {});
  struct EF { uint32_t a, b; uint64_t f; };
  std::vector<char> vis(q.n, 0);
  vis[root] = 1;
  std::vector<EF> cur;
  for (uint32_t w : q.nbr[root]) cur.push_back({root, w, freq[root][w]});
  while (!cur.empty()) {
    std::vector<EF> next;
    while (!cur.empty()) {
      size_t best = 0;
      for (size_t i = 1; i < cur.size(); i++) if (cur[i].f < cur[best].f) best = i;
      const EF m = cur[best];
      std::vector<EF> keep;
      for (const EF& e : cur) if (e.b != m.b) keep.push_back(e);
      cur.swap(keep);
      if (vis[m.b]) continue;
      vis[m.b] = 1;
      const uint32_t l = q.edge_label(m.a, m.b);
      d.chd[m.a].push_back(m.b); d.chd_l[m.a].push_back(l);
      d.par[m.b].push_back(m.a); d.par_l[m.b].push_back(l);
      for (uint32_t w : q.nbr[m.b]) if (!vis[w]) next.push_back({m.b, w, freq[m.b][w]});
    }
    cur.swap(next);
  }
  d.order.clear();
  std::vector<uint32_t> fifo{root};
  for (size_t h = 0; h < fifo.size(); h++) {
    d.order.push_back(fifo[h]);
    for (uint32_t w : d.chd[fifo[h]]) fifo.push_back(w);
  }
}

bool has_support(const Graph& g, uint32_t v, uint32_t lab, uint32_t el, const std::vector<char>& flag) {
  for (size_t j = 0; j < g.nbr[v].size(); j++) {
    const uint32_t w = g.nbr[v][j];
    if (g.elab[v][j] == el && g.label(w) == lab && flag[w]) return true;
  }
  return false;
}

// d1 / d2 flags by their definition (symbi.cpp:259-349; the counters n1,
// np1, n2, nc2 of InsertionTopDown ... DeletionBottomUp, symbi.cpp:404-469,
// maintain the same fixpoint under updates):
//   d1[u][v]: L(v) = L(u) and every DAG parent p has a neighbour w of v over
//             an edge labelled l(u, p) with d1[p][w];
//   d2[u][v]: d1[u][v] and every DAG child c has a neighbour w of v over an
//             edge labelled l(u, c) with d2[c][w].
void dag_flags(const QueryGraph& q, const Graph& g, const Dag& d, std::vector<std::vector<char>>& d1,
               std::vector<std::vector<char>>& d2) {
  const size_t n = g.vlabel.size();
  d1.assign(q.n, std::vector<char>(n, 0));
  d2.assign(q.n, std::vector<char>(n, 0));
  for (uint32_t u : d.order)
    for (uint32_t v = 0; v < n; v++) {
      if (g.vlabel[v] == NOT_EXIST || g.vlabel[v] != q.vlabel[u]) continue;
      bool ok = true;
      for (size_t k = 0; k < d.par[u].size() && ok; k++)
        ok = has_support(g, v, q.vlabel[d.par[u][k]], d.par_l[u][k], d1[d.par[u][k]]);
      d1[u][v] = ok;
    }
  for (size_t i = d.order.size(); i-- > 0;) {
    const uint32_t u = d.order[i];
    for (uint32_t v = 0; v < n; v++) {
      if (!d1[u][v]) continue;
      bool ok = true;
      for (size_t k = 0; k < d.chd[u].size() && ok; k++)
        ok = has_support(g, v, q.vlabel[d.chd[u][k]], d.chd_l[u][k], d2[d.chd[u][k]]);
      d2[u][v] = ok;
    }
  }
}

}  // namespace

extern "C" int oracle_index(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                            uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
                            uint64_t n_up, const oracle_update* ups, int algo, uint32_t* root, uint32_t* order,
                            uint32_t* parents, uint64_t words, uint64_t* d1_out, uint64_t* d2_out) {
  QueryGraph q;
  if (n_qv < 2 || n_qv > 32 || !q.build(n_qv, q_vlabels, n_qe, q_edges) || q.n_edges == 0) return -1;
  if (algo != ORACLE_INDEX_TURBOFLUX && algo != ORACLE_INDEX_SYMBI) return -2;
  Graph g;
  for (uint32_t v = 0; v < n_v; v++) g.add_vertex(v, vlabels[v]);
  if (g.vlabel.size() < n_v) { g.vlabel.resize(n_v, NOT_EXIST); g.nbr.resize(n_v); g.elab.resize(n_v); }
  for (uint64_t i = 0; i < n_e; i++) {
    uint32_t a = edges[3 * i], b = edges[3 * i + 1];
    if (a < n_v && b < n_v && a != b) g.add_edge(a, b, edges[3 * i + 2]);
  }
  // the DAG is fixed at preprocessing, on the graph before the stream
  std::vector<std::vector<uint64_t>> freq;
  const uint32_t r = dag_root(q, g, freq);
  Dag d;
  if (algo == ORACLE_INDEX_SYMBI) dag_symbi(q, r, d); else dag_turboflux(q, r, freq, d);
  for (uint64_t i = 0; i < n_up; i++) {  // the graph after the stream prefix
    const oracle_update& u = ups[i];
    if (u.type == 'v') {
      if (u.is_add) g.add_vertex(u.id1, u.label);
      else if (u.id1 < g.vlabel.size()) {
        std::vector<uint32_t> ns = g.nbr[u.id1];
        for (uint32_t w : ns) g.remove_edge(u.id1, w);
        g.vlabel[u.id1] = NOT_EXIST;
      }
      continue;
    }
    if (u.id1 >= g.vlabel.size() || u.id2 >= g.vlabel.size() || u.id1 == u.id2) continue;
    if (u.is_add) g.add_edge(u.id1, u.id2, u.label); else g.remove_edge(u.id1, u.id2);
  }
  const size_t n = g.vlabel.size();
  if (words * 64 < n) return -3;
  std::vector<std::vector<char>> d1, d2;
  dag_flags(q, g, d, d1, d2);
  *root = d.root;
  for (uint32_t i = 0; i < n_qv; i++) order[i] = d.order[i];
  for (uint32_t u = 0; u < n_qv; u++) {
    uint32_t m = 0;
    for (uint32_t p : d.par[u]) m |= 1u << p;
    parents[u] = m;
    for (uint64_t w = 0; w < words; w++) { d1_out[u * words + w] = 0; d2_out[u * words + w] = 0; }
    for (size_t v = 0; v < n; v++) {
      if (d1[u][v]) d1_out[u * words + (v >> 6)] |= 1ULL << (v & 63);
      if (d2[u][v]) d2_out[u * words + (v >> 6)] |= 1ULL << (v & 63);
    }
  }
  return (int)n;
}

namespace {

// Can the query neighbours of u be mapped to distinct neighbours w of v, each
// over an edge with the query edge's label, onto a vertex with the query
// neighbour's label and lit[uj][w]?  (Without injectivity under homo.)
// Augmenting paths over the query side (at most 31 neighbours).
bool calig_inject(const QueryGraph& q, const Graph& g, uint32_t u, uint32_t v,
                  const std::vector<std::vector<char>>& lit, bool homo) {
  const auto& qn = q.nbr[u];
  const auto& ql = q.elab[u];
  const auto& dn = g.nbr[v];
  const auto& dl = g.elab[v];
  auto fits = [&](size_t i, size_t j) {
    const uint32_t uj = qn[i], w = dn[j];
    return dl[j] == ql[i] && g.label(w) == q.vlabel[uj] && lit[uj][w];
  };
  if (homo) {
    for (size_t i = 0; i < qn.size(); i++) {
      bool any = false;
      for (size_t j = 0; j < dn.size() && !any; j++) any = fits(i, j);
      if (!any) return false;
    }
    return true;
  }
  if (qn.size() > dn.size()) return false;
  std::vector<int> owner(dn.size(), -1);  // data neighbour -> query neighbour index
  for (size_t i = 0; i < qn.size(); i++) {
    std::vector<char> seen(dn.size(), 0);
    std::function<bool(size_t)> augment = [&](size_t a) {
      for (size_t j = 0; j < dn.size(); j++) {
        if (seen[j] || !fits(a, j)) continue;
        seen[j] = 1;
        if (owner[j] < 0 || augment((size_t)owner[j])) { owner[j] = (int)a; return true; }
      }
      return false;
    };
    if (!augment(i)) return false;
  }
  return true;
}

// The lighting of CaLiG after static filtering (constructCand + staticFilter,
// ParaCOSM/CSM/matching/Parallel_CaLiG/parallel_calig.cpp:337-361, 385-396,
// 398-429, 970-975): the greatest set of (u, v) pairs with L(v) = L(u) such
// that every lit (u, v) can map u's query neighbours to distinct lit
// neighbours of v.  The reference checks one candidate per neighbour
// (checkNei) plus distinct witnesses inside each group of same-label
// neighbours (tryNei over rep_nei); witnesses of different labels are
// distinct anyway, so that is one injective map of the whole neighbourhood.
void calig_fixpoint(const QueryGraph& q, const Graph& g, bool homo, std::vector<std::vector<char>>& lit) {
  const size_t n = g.vlabel.size();
  lit.assign(q.n, std::vector<char>(n, 0));
  for (uint32_t u = 0; u < q.n; u++)
    for (size_t v = 0; v < n; v++) lit[u][v] = g.vlabel[v] != NOT_EXIST && g.vlabel[v] == q.vlabel[u];
  for (bool changed = true; changed;) {
    changed = false;
    for (uint32_t u = 0; u < q.n; u++)
      for (uint32_t v = 0; v < n; v++)
        if (lit[u][v] && !calig_inject(q, g, u, v, lit, homo)) { lit[u][v] = 0; changed = true; }
  }
}

// The two bounded levels the engine maintains for its CaLiG-style plugin
// (a sound superset of the lighting above, exact under every update):
//   li0[u][v]: L(v) = L(u) and, for every (vertex label, edge label) pair c
//              of u's query edges, v has at least as many neighbours of
//              pair c as u has (one under homo);
//   li1[u][v]: li0[u][v] and every query neighbour uj of u has a neighbour w
//              of v over an edge labelled l(u, uj) with li0[uj][w].
void calig_levels(const QueryGraph& q, const Graph& g, bool homo, std::vector<std::vector<char>>& li0,
                  std::vector<std::vector<char>>& li1) {
  const size_t n = g.vlabel.size();
  li0.assign(q.n, std::vector<char>(n, 0));
  li1.assign(q.n, std::vector<char>(n, 0));
  for (uint32_t u = 0; u < q.n; u++) {
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> need;
    for (size_t i = 0; i < q.nbr[u].size(); i++) need[{q.vlabel[q.nbr[u][i]], q.elab[u][i]}]++;
    for (size_t v = 0; v < n; v++) {
      if (g.vlabel[v] == NOT_EXIST || g.vlabel[v] != q.vlabel[u]) continue;
      bool ok = true;
      for (const auto& kv : need) {
        uint32_t have = 0;
        for (size_t j = 0; j < g.nbr[v].size(); j++)
          if (g.elab[v][j] == kv.first.second && g.label(g.nbr[v][j]) == kv.first.first) have++;
        if (have < (homo ? 1u : kv.second)) { ok = false; break; }
      }
      li0[u][v] = ok;
    }
  }
  for (uint32_t u = 0; u < q.n; u++)
    for (uint32_t v = 0; v < n; v++) {
      if (!li0[u][v]) continue;
      bool ok = true;
      for (size_t i = 0; i < q.nbr[u].size() && ok; i++)
        ok = has_support(g, v, q.vlabel[q.nbr[u][i]], q.elab[u][i], li0[q.nbr[u][i]]);
      li1[u][v] = ok;
    }
}

void pack_bits(const std::vector<std::vector<char>>& f, uint64_t words, uint64_t* out) {
  for (size_t u = 0; u < f.size(); u++) {
    for (uint64_t w = 0; w < words; w++) out[u * words + w] = 0;
    for (size_t v = 0; v < f[u].size(); v++)
      if (f[u][v]) out[u * words + (v >> 6)] |= 1ULL << (v & 63);
  }
}

}  // namespace

extern "C" uint64_t oracle_group_assignments(uint32_t g, const uint64_t* N, int homo) {
  if (g == 0 || g > kTailGroup) return 0;
  uint64_t n[1u << kTailGroup] = {0};
  for (uint32_t M = 1; M < (1u << g); M++) n[M] = N[M];
  return group_assignments(g, n, homo != 0);
}

extern "C" int oracle_calig_index(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                                  uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
                                  uint64_t n_up, const oracle_update* ups, int homo, uint64_t words, uint64_t* li0_out,
                                  uint64_t* li1_out, uint64_t* lit_out) {
  QueryGraph q;
  if (n_qv < 2 || n_qv > 32 || !q.build(n_qv, q_vlabels, n_qe, q_edges) || q.n_edges == 0) return -1;
  Graph g;
  for (uint32_t v = 0; v < n_v; v++) g.add_vertex(v, vlabels[v]);
  if (g.vlabel.size() < n_v) { g.vlabel.resize(n_v, NOT_EXIST); g.nbr.resize(n_v); g.elab.resize(n_v); }
  for (uint64_t i = 0; i < n_e; i++) {
    uint32_t a = edges[3 * i], b = edges[3 * i + 1];
    if (a < n_v && b < n_v && a != b) g.add_edge(a, b, edges[3 * i + 2]);
  }
  for (uint64_t i = 0; i < n_up; i++) {
    const oracle_update& u = ups[i];
    if (u.type == 'v') {
      if (u.is_add) g.add_vertex(u.id1, u.label);
      else if (u.id1 < g.vlabel.size()) {
        std::vector<uint32_t> ns = g.nbr[u.id1];
        for (uint32_t w : ns) g.remove_edge(u.id1, w);
        g.vlabel[u.id1] = NOT_EXIST;
      }
      continue;
    }
    if (u.id1 >= g.vlabel.size() || u.id2 >= g.vlabel.size() || u.id1 == u.id2) continue;
    if (u.is_add) g.add_edge(u.id1, u.id2, u.label); else g.remove_edge(u.id1, u.id2);
  }
  const size_t n = g.vlabel.size();
  if (words * 64 < n) return -3;
  std::vector<std::vector<char>> li0, li1, lit;
  calig_levels(q, g, homo != 0, li0, li1);
  if (li0_out) pack_bits(li0, words, li0_out);
  if (li1_out) pack_bits(li1, words, li1_out);
  if (lit_out) {
    calig_fixpoint(q, g, homo != 0, lit);
    pack_bits(lit, words, lit_out);
  }
  return (int)n;
}

// InitialMatching (ParaCOSM/CSM/matching/GraphFlow/graphflow.cpp:268-284):
// every vertex with the label of the first vertex of order 0 starts a
// FindMatches from depth 1; no per-update cap.  Counted on the graph after
// the first n_up updates.
extern "C" int oracle_initial_count(uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges,
                                    uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges,
                                    uint64_t n_up, const oracle_update* ups, int homo, uint64_t* count) {
  QueryGraph q;
  if (n_qv < 2 || !q.build(n_qv, q_vlabels, n_qe, q_edges) || q.n_edges == 0) return -1;
  Graph g;
  for (uint32_t v = 0; v < n_v; v++) g.add_vertex(v, vlabels[v]);
  if (g.vlabel.size() < n_v) { g.vlabel.resize(n_v, NOT_EXIST); g.nbr.resize(n_v); g.elab.resize(n_v); }
  for (uint64_t i = 0; i < n_e; i++) {
    uint32_t a = edges[3 * i], b = edges[3 * i + 1];
    if (a < n_v && b < n_v && a != b) g.add_edge(a, b, edges[3 * i + 2]);
  }
  for (uint64_t i = 0; i < n_up; i++) {
    const oracle_update& u = ups[i];
    if (u.type == 'v') { if (u.is_add) g.add_vertex(u.id1, u.label); continue; }
    if (u.id1 >= g.vlabel.size() || u.id2 >= g.vlabel.size() || u.id1 == u.id2) continue;
    if (u.is_add) g.add_edge(u.id1, u.id2, u.label); else g.remove_edge(u.id1, u.id2);
  }
  std::vector<std::vector<uint32_t>> order;
  graphflow_orders(q, order);
  Searcher s(q, g, order, homo != 0, false, 0);
  s.m.assign(n_qv, NOT_EXIST);
  s.visited.assign(g.vlabel.size(), 0);
  const uint32_t u0 = order[0][0];
  for (uint32_t v = 0; v < g.vlabel.size(); v++) {
    if (g.vlabel[v] == NOT_EXIST || g.vlabel[v] != q.vlabel[u0]) continue;
    s.m[u0] = v; s.visited[v] = 1;
    s.find(0, 1, 0);
    s.visited[v] = 0; s.m[u0] = NOT_EXIST;
  }
  *count = s.count;
  return 0;
}
