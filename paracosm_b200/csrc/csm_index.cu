// Candidate index of the TurboFlux / SymBi plugins (meaning and layout in
// csm_index.cuh).
//
// Kernels (all integer work, bound by L2/HBM latency of the segment reads):
//   k_ix_freq   query-edge frequencies and label counts that choose the root
//               (ParaCOSM/CSM/matching/SymBi/symbi.cpp:116-195)
//   k_ix_seed   marks the endpoints of changed directed entries for
//               re-evaluation (the reference's per-edge Insertion/Deletion
//               TopDown/BottomUp entry, symbi.cpp:679-735)
//   k_ix_prop   marks the DAG-neighbour-side neighbours of vertices whose
//               flag changed (the Q1 / Q2 propagation loops, symbi.cpp:714-735)
//   k_ix_eval   re-evaluates marked flags of one query vertex from their
//               definition: one warp per 64-vertex word; short segments are
//               scanned by one lane each, long ones by the whole warp with
//               an early exit on the first supporting neighbour
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>

#include "csm_index.cuh"

namespace cg = cooperative_groups;

namespace csm {

namespace {

constexpr uint32_t kLaneScanMax = 48;  // entries a single lane scans before handing a vertex to the warp

__device__ __forceinline__ bool bit_of(const uint64_t* a, uint32_t v) { return (a[v >> 6] >> (v & 63)) & 1ULL; }

__device__ __forceinline__ uint64_t warp_or64(uint64_t x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x |= __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Does some neighbour w in segment [lo, hi) of the pool have flag[w]?  One lane.
__device__ __forceinline__ bool lane_support(const uint32_t* pool, uint64_t lo, uint64_t hi, const uint64_t* flag) {
  for (uint64_t k = lo; k < hi; k++)
    if (bit_of(flag, pool[k])) return true;
  return false;
}

// Entries of v in combo c (the union graph's segment during a batch).
__device__ __forceinline__ uint64_t seg_count(const DevGraph& g, uint32_t v, uint32_t c) {
  uint64_t lo, hi;
  segment(g, v, c, lo, hi);
  return hi - lo;
}

// The same over the whole warp (every lane must call it with equal arguments).
__device__ __forceinline__ bool warp_support(const uint32_t* pool, uint64_t lo, uint64_t hi, const uint64_t* flag,
                                             uint32_t lane) {
  for (uint64_t b = lo; b < hi; b += 32) {
    const uint64_t k = b + lane;
    const bool hit = k < hi && bit_of(flag, pool[k]);
    if (__any_sync(0xffffffffu, hit)) return true;
  }
  return false;
}

}  // namespace

// Per query edge (u < u' in adjacency order): directed entries v -> v' with
// L(v) = L(u), L(v') = L(u') and the edge's label = sum over v of L(u) of the
// segment size S(v, L(u'), l).  Also the number of vertices per folded label.
__global__ void k_ix_freq(DevGraph g, uint32_t ne, const uint32_t* __restrict__ eu, const uint32_t* __restrict__ ecombo,
                          const uint32_t* __restrict__ elab_u, unsigned long long* freq, unsigned long long* lcount) {
  __shared__ unsigned long long s_freq[kMaxQE];
  __shared__ unsigned long long s_lc[kMaxQ + 1];
  for (uint32_t i = threadIdx.x; i < ne; i += blockDim.x) s_freq[i] = 0;
  for (uint32_t i = threadIdx.x; i <= kMaxQ; i += blockDim.x) s_lc[i] = 0;
  __syncthreads();
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += gridDim.x * blockDim.x) {
    const uint32_t lv = g.vlabel[v];
    if (lv == kNone) continue;
    if (lv <= kMaxQ) atomicAdd(&s_lc[lv], 1ull);
    const uint32_t* d = g.dir + (size_t)v * (g.nc + 1);
    for (uint32_t e = 0; e < ne; e++) {
      if (elab_u[e] != lv) continue;
      const uint32_t c = ecombo[e];
      const uint32_t sz = d[c + 1] - d[c];
      if (sz) atomicAdd(&s_freq[e], (unsigned long long)sz);
    }
  }
  (void)eu;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < ne; i += blockDim.x)
    if (s_freq[i]) atomicAdd(&freq[i], s_freq[i]);
  for (uint32_t i = threadIdx.x; i <= kMaxQ; i += blockDim.x)
    if (s_lc[i]) atomicAdd(&lcount[i], s_lc[i]);
}

// Marks, for every changed directed entry x -> y (combo = (L(y), l)) and every
// DAG edge p -> c with L(p) = L(x), L(c) = L(y) and label l: y for d1 of c,
// x for d2 of p.  The reverse entry y -> x covers the other orientation.
__global__ void k_ix_seed(const uint64_t* __restrict__ keys, uint32_t L, DevGraph g, const IxDag* __restrict__ dag,
                          IxBits b) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L) return;
  const uint64_t k = keys[i];
  if (!g.kb.real(k)) return;
  const uint32_t x = g.kb.x_of(k), c = g.kb.c_of(k), y = g.kb.y_of(k);
  const uint32_t ly = c / g.n_el, el = c % g.n_el;
  const uint32_t lx = g.vlabel[x];
  const uint32_t ne = dag->n_edges;
  for (uint32_t e = 0; e < ne; e++) {
    if (dag->eel[e] != el) continue;
    const uint32_t p = dag->ep[e], ch = dag->ec[e];
    if (dag->qlab[p] != lx || dag->qlab[ch] != ly) continue;
    atomicOr((unsigned long long*)&b.m1[(uint64_t)ch * b.words + (y >> 6)], 1ull << (y & 63));
    atomicOr((unsigned long long*)&b.m2[(uint64_t)p * b.words + (x >> 6)], 1ull << (x & 63));
    *b.active = 1u;
  }
}

// A new vertex: mark it for every query vertex (only its d1 at the root can
// become set; the evaluation decides).
__global__ void k_ix_seed_vertex(uint32_t v, const IxDag* __restrict__ dag, IxBits b) {
  const uint32_t u = threadIdx.x;
  if (u >= dag->nq) return;
  if (u == 0) *b.active = 1u;
  b.m1[(uint64_t)u * b.words + (v >> 6)] |= 1ull << (v & 63);
  b.m2[(uint64_t)u * b.words + (v >> 6)] |= 1ull << (v & 63);
}

// Phase 1 (d1 of u): for each parent p, every vertex w whose d1[p] changed
// marks its neighbours in S(w, L(u), l(u,p)).  Phase 2 (d2 of u): the same
// from each child c through d2[c] changes.  One warp per word of changes.
__device__ __forceinline__ void ix_prop(const DevGraph& g, const IxDag* __restrict__ dag, const IxBits& b, uint32_t u,
                                        uint32_t phase, uint32_t lane, uint32_t warp, uint32_t nwarps) {
  const uint32_t* pool = g.pools[g.ps->active];
  const uint32_t nsrc = phase == 1 ? dag->npar[u] : dag->nchd[u];
  uint64_t* dst = (phase == 1 ? b.m1 : b.m2) + (uint64_t)u * b.words;
  for (uint32_t s = 0; s < nsrc; s++) {
    const uint32_t q = phase == 1 ? dag->par[u][s] : dag->chd[u][s];
    const uint32_t combo = phase == 1 ? dag->par_ucombo[u][s] : dag->chd_ucombo[u][s];
    const uint64_t* src = (phase == 1 || dag->lighting ? b.c1 : b.c2) + (uint64_t)q * b.words;
    for (uint64_t wi = warp; wi < b.words; wi += nwarps) {
      uint64_t word = src[wi];
      while (word) {
        const uint32_t w = (uint32_t)(wi * 64 + (uint64_t)(__ffsll((long long)word) - 1));
        word &= word - 1;
        uint64_t lo, hi;
        segment(g, w, combo, lo, hi);
        for (uint64_t k = lo + lane; k < hi; k += 32) {
          const uint32_t v = pool[k];
          atomicOr((unsigned long long*)&dst[v >> 6], 1ull << (v & 63));
        }
      }
    }
  }
}

__global__ void k_ix_prop(DevGraph g, const IxDag* __restrict__ dag, IxBits b, uint32_t u, uint32_t phase) {
  if (!*b.active) return;
  ix_prop(g, dag, b, u, phase, threadIdx.x & 31, (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
          (gridDim.x * blockDim.x) >> 5);
}

// Re-evaluates the marked flags of query vertex u (phase 1: d1, phase 2: d2).
// full = 1 evaluates every vertex of u's label (index build).  Each warp owns
// whole words of the target bitset, so its updates need no atomics.
__device__ __forceinline__ void ix_eval(const DevGraph& g, const IxDag* __restrict__ dag, const IxBits& b, uint32_t u,
                                        uint32_t phase, uint32_t full, uint32_t lane, uint32_t warp,
                                        uint32_t nwarps) {
  const uint32_t* pool = g.pools[g.ps->active];
  const uint32_t lu = dag->qlab[u];
  const uint64_t off = (uint64_t)u * b.words;
  uint64_t* target = (phase == 1 ? b.d1 : b.d2) + off;
  uint64_t* mark = (phase == 1 ? b.m1 : b.m2) + off;
  uint64_t* chg = (phase == 1 ? b.c1 : b.c2) + off;
  const uint64_t* d1u = b.d1 + off;
  const uint32_t nchk = phase == 1 ? dag->npar[u] : dag->nchd[u];
  // support flags of the checked neighbours: d1 of parents; d2 of children,
  // or their d1 in lighting mode
  const uint64_t* sup = (phase == 1 || dag->lighting) ? b.d1 : b.d2;
  const uint32_t nreq = (phase == 1 && dag->lighting) ? dag->nreq[u] : 0u;
  for (uint64_t wi = warp; wi < b.words; wi += nwarps) {
    uint64_t cand;
    if (full) {
      if (phase == 1) {
        const uint64_t v0 = wi * 64 + lane, v1 = v0 + 32;
        const bool a = v0 < g.n && g.vlabel[v0] == lu;
        const bool c = v1 < g.n && g.vlabel[v1] == lu;
        cand = (uint64_t)__ballot_sync(0xffffffffu, a) | ((uint64_t)__ballot_sync(0xffffffffu, c) << 32);
      } else {
        cand = d1u[wi];
      }
    } else {
      cand = mark[wi];
      if (phase == 2) cand |= b.c1[off + wi];
      __syncwarp();
      if (cand && lane == 0) mark[wi] = 0;
    }
    if (!cand) continue;
    const uint64_t old = target[wi];
    // pass 1: one candidate per lane (the j-th set bit goes to lane j % 32)
    uint64_t mine = 0, defer = 0;
    {
      uint64_t rest = cand;
      uint32_t j = 0;
      while (rest) {
        const uint32_t bitpos = (uint32_t)(__ffsll((long long)rest) - 1);
        rest &= rest - 1;
        if ((j++ & 31) != lane) continue;
        const uint32_t v = (uint32_t)(wi * 64 + bitpos);
        bool ok;
        bool long_seg = false;
        if (phase == 1) ok = g.vlabel[v] == lu;
        else ok = bit_of(d1u, v);
        for (uint32_t r = 0; r < nreq && ok; r++) ok = seg_count(g, v, dag->req_combo[u][r]) >= dag->req_mult[u][r];
        for (uint32_t s = 0; s < nchk && ok; s++) {
          const uint32_t q = phase == 1 ? dag->par[u][s] : dag->chd[u][s];
          const uint32_t combo = phase == 1 ? dag->par_vcombo[u][s] : dag->chd_vcombo[u][s];
          const uint64_t* flag = sup + (uint64_t)q * b.words;
          uint64_t lo, hi;
          segment(g, v, combo, lo, hi);
          if (hi - lo > kLaneScanMax) { long_seg = true; break; }
          ok = lane_support(pool, lo, hi, flag);
        }
        if (long_seg) defer |= 1ull << bitpos;
        else if (ok) mine |= 1ull << bitpos;
      }
    }
    uint64_t newbits = warp_or64(mine);
    defer = warp_or64(defer);
    // pass 2: vertices with a long segment, by the whole warp
    while (defer) {
      const uint32_t bitpos = (uint32_t)(__ffsll((long long)defer) - 1);
      defer &= defer - 1;
      const uint32_t v = (uint32_t)(wi * 64 + bitpos);
      bool ok = phase == 1 ? (g.vlabel[v] == lu) : bit_of(d1u, v);
      for (uint32_t r = 0; r < nreq && ok; r++) ok = seg_count(g, v, dag->req_combo[u][r]) >= dag->req_mult[u][r];
      for (uint32_t s = 0; s < nchk && ok; s++) {
        const uint32_t q = phase == 1 ? dag->par[u][s] : dag->chd[u][s];
        const uint32_t combo = phase == 1 ? dag->par_vcombo[u][s] : dag->chd_vcombo[u][s];
        const uint64_t* flag = sup + (uint64_t)q * b.words;
        uint64_t lo, hi;
        segment(g, v, combo, lo, hi);
        ok = warp_support(pool, lo, hi, flag, lane);
      }
      if (ok) newbits |= 1ull << bitpos;
    }
    const uint64_t nw = (old & ~cand) | (newbits & cand);
    if (lane == 0 && nw != old) {
      target[wi] = nw;
      chg[wi] |= nw ^ old;
    }
    __syncwarp();
  }
}

__global__ void k_ix_eval(DevGraph g, const IxDag* __restrict__ dag, IxBits b, uint32_t u, uint32_t phase,
                          uint32_t full) {
  if (!*b.active) return;
  ix_eval(g, dag, b, u, phase, full, threadIdx.x & 31, (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
          (gridDim.x * blockDim.x) >> 5);
}

// End of a round: the change bitsets start the next round empty.
__global__ void k_ix_clear_changes(IxBits b, uint64_t n) {
  if (!*b.active) return;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    b.c1[i] = 0;
    b.c2[i] = 0;
  }
}

// One incremental round over every query vertex in a single launch, for the
// changes of one edge update (the plain form): the steps of
// index_launch_round -- per query vertex in DAG order, propagation of the
// parents' d1 changes and re-evaluation of d1, then in reverse order the
// children's d2 changes and d2 -- separated by grid-wide barriers instead of
// kernel boundaries.  Launched cooperatively (every block resident), with a
// grid no larger than the occupancy allows.  Every block takes the same
// branches, so every block reaches every barrier.
__global__ void __launch_bounds__(256) k_ix_round_coop(DevGraph g, const IxDag* __restrict__ dag, IxBits b,
                                                       IxOrder ord) {
  if (!*b.active) return;  // nothing that the flags depend on changed: the same in every block
  cg::grid_group grid = cg::this_grid();
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = 0; i < ord.nq; i++) {
    const uint32_t u = ord.order[i];
    if (dag->npar[u] != 0) {  // the root's d1 is its label test: only new vertices change it
      ix_prop(g, dag, b, u, 1, lane, warp, nwarps);
      grid.sync();
    }
    ix_eval(g, dag, b, u, 1, 0, lane, warp, nwarps);
    grid.sync();
  }
  for (uint32_t i = ord.nq; i-- > 0;) {
    const uint32_t u = ord.order[i];
    if (dag->nchd[u] != 0) {
      ix_prop(g, dag, b, u, 2, lane, warp, nwarps);
      grid.sync();
    }
    ix_eval(g, dag, b, u, 2, 0, lane, warp, nwarps);
    grid.sync();
  }
  const uint64_t n = (uint64_t)ord.nq * b.words;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    b.c1[i] = 0;
    b.c2[i] = 0;
  }
}

__global__ void k_ix_popcount(const uint64_t* a, uint64_t n, unsigned long long* out) {
  unsigned long long s = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    s += (unsigned long long)__popcll(a[i]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

// ------------------------------------------------------------------ host

namespace {

#define IXCK(x)                                                                              \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess) return set_err(CSM_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

// Root choice (ParaCOSM/CSM/matching/SymBi/symbi.cpp:116-195, identical in
// TurboFlux/turboflux.cpp:82-149): the first query edge (u < u', adjacency
// order) of least frequency; of its endpoints the one whose label is rarer in
// the data graph, ties to the larger query degree, then to the second one.
uint32_t choose_root(const IndexQuery& q, const std::vector<std::pair<uint32_t, uint32_t>>& edges,
                     const std::vector<unsigned long long>& freq, const std::vector<unsigned long long>& lcount) {
  size_t best = 0;
  for (size_t i = 1; i < edges.size(); i++)
    if (freq[i] < freq[best]) best = i;
  const uint32_t a = edges[best].first, b = edges[best].second;
  const auto& ql = *q.vlabels;
  const unsigned long long ca = ql[a] <= kMaxQ ? lcount[ql[a]] : 0, cb = ql[b] <= kMaxQ ? lcount[ql[b]] : 0;
  if (ca > cb) return b;
  if (ca < cb) return a;
  return (*q.nbr)[a].size() > (*q.nbr)[b].size() ? a : b;
}

}  // namespace

static int index_launch_round(IndexState& ix, const DevGraph& g, cudaStream_t st, uint64_t* launches, bool full) {
  const uint32_t nq = ix.h_dag.nq;
  const uint64_t warps_needed = std::max<uint64_t>(ix.words, 1);
  const uint32_t blocks = (uint32_t)std::min<uint64_t>((warps_needed + 7) / 8, (uint64_t)ix.sm_count * 8);
  for (uint32_t i = 0; i < nq; i++) {
    const uint32_t u = ix.order[i];
    if (!full && ix.h_dag.npar[u] == 0) {
      // the root's d1 is its label test: only new vertices change it
      k_ix_eval<<<blocks, 256, 0, st>>>(g, ix.d_dag, ix.bits, u, 1, 0);
      (*launches)++;
      continue;
    }
    if (!full) { k_ix_prop<<<blocks, 256, 0, st>>>(g, ix.d_dag, ix.bits, u, 1); (*launches)++; }
    k_ix_eval<<<blocks, 256, 0, st>>>(g, ix.d_dag, ix.bits, u, 1, full ? 1u : 0u);
    (*launches)++;
  }
  for (uint32_t i = nq; i-- > 0;) {
    const uint32_t u = ix.order[i];
    if (!full && ix.h_dag.nchd[u]) { k_ix_prop<<<blocks, 256, 0, st>>>(g, ix.d_dag, ix.bits, u, 2); (*launches)++; }
    k_ix_eval<<<blocks, 256, 0, st>>>(g, ix.d_dag, ix.bits, u, 2, full ? 1u : 0u);
    (*launches)++;
  }
  k_ix_clear_changes<<<ix.sm_count * 2, 256, 0, st>>>(ix.bits, (uint64_t)nq * ix.words);
  (*launches)++;
  IXCK(cudaGetLastError());
  return CSM_OK;
}

// DAG of the TurboFlux / SymBi plugin: root from the device edge frequencies,
// then the SymBi BFS orientation or the TurboFlux spanning tree.
static int dag_for(const IndexQuery& q, const DevGraph& g, int algo,
                   const std::vector<std::pair<uint32_t, uint32_t>>& edges, const std::vector<uint32_t>& e_lab,
                   int sm_count, DevMem& mem, cudaStream_t st, uint64_t* launches, uint32_t& root,
                   std::vector<std::vector<uint32_t>>& par, std::vector<std::vector<uint32_t>>& chd,
                   std::vector<std::vector<uint32_t>>& par_l, std::vector<std::vector<uint32_t>>& chd_l,
                   std::vector<uint32_t>& order) {
  const uint32_t nq = q.n;
  const auto& ql = *q.vlabels;
  const auto& nbr = *q.nbr;
  const auto& el = *q.elabel;
  const uint32_t ne = (uint32_t)edges.size();
  // frequencies on the device
  std::vector<uint32_t> h_eu(ne), h_ec(ne), h_el(ne);
  for (uint32_t i = 0; i < ne; i++) {
    h_eu[i] = edges[i].first;
    h_ec[i] = ql[edges[i].second] * g.n_el + e_lab[i];
    h_el[i] = ql[edges[i].first];
  }
  uint32_t* d_e = nullptr;
  unsigned long long* d_f = nullptr;
  int rc = mem.alloc((void**)&d_e, 12ull * ne);
  if (rc) return rc;
  rc = mem.alloc((void**)&d_f, 8ull * (ne + kMaxQ + 1));
  if (rc) { mem.release(d_e, 12ull * ne); return rc; }
  IXCK(cudaMemcpyAsync(d_e, h_eu.data(), 4ull * ne, cudaMemcpyHostToDevice, st));
  IXCK(cudaMemcpyAsync(d_e + ne, h_ec.data(), 4ull * ne, cudaMemcpyHostToDevice, st));
  IXCK(cudaMemcpyAsync(d_e + 2 * ne, h_el.data(), 4ull * ne, cudaMemcpyHostToDevice, st));
  IXCK(cudaMemsetAsync(d_f, 0, 8ull * (ne + kMaxQ + 1), st));
  k_ix_freq<<<sm_count * 4, 256, 0, st>>>(g, ne, d_e, d_e + ne, d_e + 2 * ne, d_f, d_f + ne);
  (*launches)++;
  IXCK(cudaGetLastError());
  std::vector<unsigned long long> freq(ne + kMaxQ + 1);
  IXCK(cudaMemcpyAsync(freq.data(), d_f, 8ull * (ne + kMaxQ + 1), cudaMemcpyDeviceToHost, st));
  IXCK(cudaStreamSynchronize(st));
  mem.release(d_e, 12ull * ne);
  mem.release(d_f, 8ull * (ne + kMaxQ + 1));
  std::vector<unsigned long long> lcount(freq.begin() + ne, freq.end());
  freq.resize(ne);
  root = choose_root(q, edges, freq, lcount);

  // the DAG: parents / children with edge labels
  auto ffreq = [&](uint32_t a, uint32_t b) {
    const uint32_t x = std::min(a, b), y = std::max(a, b);
    for (uint32_t i = 0; i < ne; i++)
      if (edges[i].first == x && edges[i].second == y) return freq[i];
    return 0ull;
  };
  auto qlabel_of = [&](uint32_t a, uint32_t b) {
    auto it = std::lower_bound(nbr[a].begin(), nbr[a].end(), b);
    return el[a][(size_t)(it - nbr[a].begin())];
  };
  if (algo == CSM_ALGO_SYMBI) {
    // BFS from the root over every query edge; an edge points from the
    // endpoint dequeued first (symbi.cpp:197-238)
    std::vector<char> seen(nq, 0), popped(nq, 0);
    order.push_back(root);
    seen[root] = 1;
    for (size_t h = 0; h < order.size(); h++) {
      const uint32_t u = order[h];
      popped[u] = 1;
      for (size_t i = 0; i < nbr[u].size(); i++) {
        const uint32_t w = nbr[u][i];
        if (!seen[w]) { seen[w] = 1; order.push_back(w); }
        if (!popped[w]) {
          chd[u].push_back(w); chd_l[u].push_back(el[u][i]);
          par[w].push_back(u); par_l[w].push_back(el[u][i]);
        }
      }
    }
  } else {
    // spanning tree grown level by level, cheapest pending edge first, other
    // pending edges into the chosen vertex dropped (turboflux.cpp:151-219)
    struct EF { uint32_t a, b; unsigned long long f; };
    std::vector<char> vis(nq, 0);
    vis[root] = 1;
    std::vector<EF> cur;
    for (uint32_t w : nbr[root]) cur.push_back({root, w, ffreq(root, w)});
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
        const uint32_t l = qlabel_of(m.a, m.b);
        chd[m.a].push_back(m.b); chd_l[m.a].push_back(l);
        par[m.b].push_back(m.a); par_l[m.b].push_back(l);
        for (uint32_t w : nbr[m.b]) if (!vis[w]) next.push_back({m.b, w, ffreq(m.b, w)});
      }
      cur.swap(next);
    }
    order.push_back(root);
    for (size_t h = 0; h < order.size(); h++)
      for (uint32_t w : chd[order[h]]) order.push_back(w);
  }
  return CSM_OK;
}


// Device DAG, flag bitsets and the full first evaluation.
static int index_finish(IndexState& ix, DevMem& mem, const DevGraph& g, const IndexQuery& q, int algo, uint32_t root,
                        const std::vector<uint32_t>& order, const std::vector<std::vector<uint32_t>>& par,
                        const std::vector<std::vector<uint32_t>>& chd, const std::vector<std::vector<uint32_t>>& par_l,
                        const std::vector<std::vector<uint32_t>>& chd_l, cudaStream_t st, uint64_t* launches) {
  const uint32_t nq = q.n;
  const auto& ql = *q.vlabels;
  int rc = CSM_OK;
  IxDag& D = ix.h_dag;
  memset(&D, 0, sizeof(D));
  D.nq = nq;
  for (uint32_t u = 0; u < nq; u++) D.qlab[u] = ql[u];
  for (uint32_t u = 0; u < nq; u++) {
    D.npar[u] = (uint32_t)par[u].size();
    D.nchd[u] = (uint32_t)chd[u].size();
    for (size_t i = 0; i < par[u].size(); i++) {
      const uint32_t p = par[u][i], l = par_l[u][i];
      D.par[u][i] = (uint8_t)p;
      D.par_vcombo[u][i] = (uint16_t)(ql[p] * g.n_el + l);
      D.par_ucombo[u][i] = (uint16_t)(ql[u] * g.n_el + l);
    }
    for (size_t i = 0; i < chd[u].size(); i++) {
      const uint32_t c = chd[u][i], l = chd_l[u][i];
      D.chd[u][i] = (uint8_t)c;
      D.chd_vcombo[u][i] = (uint16_t)(ql[c] * g.n_el + l);
      D.chd_ucombo[u][i] = (uint16_t)(ql[u] * g.n_el + l);
      D.ep[D.n_edges] = (uint8_t)u; D.ec[D.n_edges] = (uint8_t)c; D.eel[D.n_edges] = (uint16_t)l;
      D.n_edges++;
    }
  }
  if (algo == CSM_ALGO_CALIG || algo == CSM_ALGO_NEWSP) {
    // d1 requirements: per (vertex label, edge label) pair of u's query
    // edges, as many neighbours as u has of that pair (one under homo)
    D.lighting = 1;
    for (uint32_t u = 0; u < nq; u++)
      for (size_t i = 0; i < chd[u].size(); i++) {
        const uint16_t combo = D.chd_vcombo[u][i];
        uint32_t r = 0;
        while (r < D.nreq[u] && D.req_combo[u][r] != combo) r++;
        if (r == D.nreq[u]) { D.req_combo[u][r] = combo; D.req_mult[u][r] = 0; D.nreq[u]++; }
        if (!q.homo || D.req_mult[u][r] == 0) D.req_mult[u][r]++;
      }
  }
  ix.root = root;
  ix.order = order;

  // flag bitsets, 32-byte aligned rows
  ix.words = ((uint64_t)g.n_cap + 63) / 64;
  ix.words = (ix.words + 3) & ~3ull;
  const uint64_t fam = 8ull * nq * ix.words;
  rc = mem.alloc((void**)&ix.bits.d1, 6 * fam);
  if (rc) return rc;
  ix.bits.d2 = ix.bits.d1 + nq * ix.words;
  ix.bits.m1 = ix.bits.d2 + nq * ix.words;
  ix.bits.m2 = ix.bits.m1 + nq * ix.words;
  ix.bits.c1 = ix.bits.m2 + nq * ix.words;
  ix.bits.c2 = ix.bits.c1 + nq * ix.words;
  ix.bits.words = ix.words;
  rc = mem.alloc((void**)&ix.d_dag, sizeof(IxDag));
  if (rc) return rc;
  rc = mem.alloc((void**)&ix.d_pop, 16);
  if (rc) return rc;
  rc = mem.alloc((void**)&ix.bits.active, 16);
  if (rc) return rc;
  IXCK(cudaMemsetAsync(ix.bits.active, 0xff, 4, st));  // the build evaluates everything
  IXCK(cudaMemsetAsync(ix.bits.d1, 0, 6 * fam, st));
  IXCK(cudaMemcpyAsync(ix.d_dag, &D, sizeof(IxDag), cudaMemcpyHostToDevice, st));
  ix.d2 = ix.bits.d2;
  ix.active = true;
  rc = index_launch_round(ix, g, st, launches, true);
  if (rc) return rc;
  IXCK(cudaStreamSynchronize(st));
  return CSM_OK;
}

int index_build(IndexState& ix, DevMem& mem, const DevGraph& g, const IndexQuery& q, int algo, int sm_count,
                cudaStream_t st, uint64_t* launches) {
  index_free(ix, mem);
  ix.algo = algo;
  ix.sm_count = sm_count > 0 ? sm_count : 148;
  if (algo != CSM_ALGO_TURBOFLUX && algo != CSM_ALGO_SYMBI && algo != CSM_ALGO_CALIG && algo != CSM_ALGO_NEWSP)
    return CSM_OK;
  const bool lighting = algo == CSM_ALGO_CALIG || algo == CSM_ALGO_NEWSP;
  const uint32_t nq = q.n;
  const auto& ql = *q.vlabels;
  const auto& nbr = *q.nbr;
  const auto& el = *q.elabel;
  // query edges u < u' in adjacency order, as the frequency scan visits them
  std::vector<std::pair<uint32_t, uint32_t>> edges;
  std::vector<uint32_t> e_lab;
  for (uint32_t u = 0; u < nq; u++)
    for (size_t i = 0; i < nbr[u].size(); i++)
      if (u < nbr[u][i]) { edges.emplace_back(u, nbr[u][i]); e_lab.push_back(el[u][i]); }
  const uint32_t ne = (uint32_t)edges.size();
  if (ne == 0 || ne > kMaxQE || nq > kMaxQ) return set_err(CSM_EUNSUPPORTED, "query size outside the index limits");
  if (lighting && 2 * ne > kMaxQE)
    return set_err(CSM_EUNSUPPORTED, "query has more than %u edges (lighting filter limit)", kMaxQE / 2);
  std::vector<std::vector<uint32_t>> par(nq), chd(nq), par_l(nq), chd_l(nq);
  std::vector<uint32_t> order;
  uint32_t root = 0;
  if (lighting) {
    // lighting: every query neighbour is a child, nobody has a parent
    for (uint32_t u = 0; u < nq; u++) {
      order.push_back(u);
      for (size_t i = 0; i < nbr[u].size(); i++) { chd[u].push_back(nbr[u][i]); chd_l[u].push_back(el[u][i]); }
    }
  } else {
    const int rc = dag_for(q, g, algo, edges, e_lab, ix.sm_count, mem, st, launches, root, par, chd, par_l, chd_l,
                           order);
    if (rc) return rc;
  }
  if (order.size() != nq) return set_err(CSM_EINVAL, "query graph is not connected");
  const int rc = index_finish(ix, mem, g, q, algo, root, order, par, chd, par_l, chd_l, st, launches);
  // the NewSP-style plugin filters candidates by the neighbour-label
  // frequencies alone (d1); d2 is still kept
  if (rc == CSM_OK && algo == CSM_ALGO_NEWSP) ix.d2 = ix.bits.d1;
  return rc;
}

// The incremental round as one cooperative launch (k_ix_round_coop).
static int index_round_coop(IndexState& ix, const DevGraph& g, cudaStream_t st, uint64_t* launches) {
  if (!ix.coop_blocks) {
    int occ = 0;
    IXCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ix_round_coop, 256, 0));
    const uint64_t warps_needed = std::max<uint64_t>(ix.words, 1);
    ix.coop_blocks = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>((warps_needed + 7) / 8, (uint64_t)ix.sm_count * (uint64_t)std::max(occ, 1)));
  }
  IxOrder ord{};
  ord.nq = ix.h_dag.nq;
  for (uint32_t i = 0; i < ord.nq; i++) ord.order[i] = ix.order[i];
  DevGraph gv = g;
  const IxDag* dag = ix.d_dag;
  IxBits bits = ix.bits;
  void* args[] = {&gv, &dag, &bits, &ord};
  IXCK(cudaLaunchCooperativeKernel((const void*)k_ix_round_coop, dim3(ix.coop_blocks), dim3(256), args, 0, st));
  (*launches)++;
  return CSM_OK;
}

// A batch's changed edges: the seed over all of them, then the round in one
// launch (2 |V_Q| + 1 launches per batch before).
int index_apply_edges(IndexState& ix, const DevGraph& g, const uint64_t* keys, uint32_t L, cudaStream_t st,
                      uint64_t* launches) {
  if (!ix.active || L == 0) return CSM_OK;
  IXCK(cudaMemsetAsync(ix.bits.active, 0, 4, st));  // set by the seed when a changed entry matters
  k_ix_seed<<<(L + 255) / 256, 256, 0, st>>>(keys, L, g, ix.d_dag, ix.bits);
  (*launches)++;
  return index_round_coop(ix, g, st, launches);
}

int index_apply_edge_one(IndexState& ix, const DevGraph& g, const uint64_t* keys, cudaStream_t st,
                         uint64_t* launches) {
  if (!ix.active) return CSM_OK;
  IXCK(cudaMemsetAsync(ix.bits.active, 0, 4, st));  // set by the seed when a changed entry matters
  k_ix_seed<<<1, 32, 0, st>>>(keys, 2, g, ix.d_dag, ix.bits);
  (*launches)++;
  return index_round_coop(ix, g, st, launches);
}

int index_vertex_update(IndexState& ix, const DevGraph& g, const csm_update& h, cudaStream_t st, uint64_t* launches) {
  if (!ix.active) return CSM_OK;
  if (h.type != 'v' || h.id1 >= g.n_cap) return CSM_OK;  // a new or a removed vertex: re-evaluate its flags
  IXCK(cudaMemsetAsync(ix.bits.active, 0, 4, st));
  k_ix_seed_vertex<<<1, 32, 0, st>>>(h.id1, ix.d_dag, ix.bits);
  (*launches)++;
  return index_launch_round(ix, g, st, launches, false);
}

int index_counts(IndexState& ix, cudaStream_t st, uint64_t* d1_count, uint64_t* d2_count) {
  *d1_count = 0; *d2_count = 0;
  if (!ix.active) return CSM_OK;
  const uint64_t n = (uint64_t)ix.h_dag.nq * ix.words;
  IXCK(cudaMemsetAsync(ix.d_pop, 0, 16, st));
  k_ix_popcount<<<ix.sm_count * 2, 256, 0, st>>>(ix.bits.d1, n, (unsigned long long*)ix.d_pop);
  k_ix_popcount<<<ix.sm_count * 2, 256, 0, st>>>(ix.bits.d2, n, (unsigned long long*)ix.d_pop + 1);
  IXCK(cudaGetLastError());
  unsigned long long h[2];
  IXCK(cudaMemcpyAsync(h, ix.d_pop, 16, cudaMemcpyDeviceToHost, st));
  IXCK(cudaStreamSynchronize(st));
  *d1_count = h[0]; *d2_count = h[1];
  ix.entries = h[0]; ix.vertices = h[1];
  return CSM_OK;
}

void index_stats(const IndexState& ix, uint64_t* entries, uint64_t* vertices) {
  *entries = ix.entries;
  *vertices = ix.vertices;
}

void index_free(IndexState& ix, DevMem& mem) {
  if (ix.bits.d1) mem.release(ix.bits.d1, 6 * 8ull * ix.h_dag.nq * ix.words);
  if (ix.d_dag) mem.release(ix.d_dag, sizeof(IxDag));
  if (ix.d_pop) mem.release(ix.d_pop, 16);
  if (ix.bits.active) mem.release(ix.bits.active, 16);
  ix.bits = IxBits{};
  ix.d_dag = nullptr;
  ix.d_pop = nullptr;
  ix.d2 = nullptr;
  ix.words = 0;
  ix.active = false;
  ix.order.clear();
}

}  // namespace csm
