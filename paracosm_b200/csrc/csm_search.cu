// Search kernels: seeding, the warp-cooperative expansion, finalisation.
//
// Reference semantics restated (paths inside ParaCOSM/CSM):
//   seeds of an edge update ......... matching/GraphFlow/graphflow.cpp:305-352 (each query
//                                     edge whose label triple matches, both orientations)
//   candidate generation / join ..... matching/GraphFlow/graphflow.cpp:181-265 (label filter,
//                                     adjacency to every matched query neighbour, injectivity)
//   index filter (TurboFlux/SymBi) .. matching/SymBi/symbi.cpp:516 (candidate must have d2 set)
//   per-update cap .................. matching/SymBi/symbi.cpp:583 (stop at exactly the cap)
//   Classify (safe update) .......... matching/Parallel_GraphFlow/parallel_graphflow.cpp:1990-2016
//
// Expansion scheme.  A warp owns one root task (update, anchor edge,
// orientation) at a time and walks its search tree depth first, but each
// level holds up to 32 partial matches at once: to extend level d the warp
// takes the next 32 (entry, driver element) pairs of level d's entries -- the
// driver being the smallest back-neighbour segment -- so lanes stay busy even
// when segments are a few elements long.  Every lane checks its candidate
// against the other back-neighbour segments (binary search), the same-label
// matched vertices (injectivity), the candidate filter, and the batch-time
// presence of every back edge; survivors are compacted with a ballot into
// level d + 1 together with the driver segment of their own next level
// (an empty next-level segment prunes them right away).  Leaves are only
// counted.
#include "csm_kernels.cuh"

namespace csm {

struct LevelSM {
  uint32_t v[32];     // data vertex of this level's position
  uint32_t dlo[32];   // driver segment of the next position: pool offset
  uint32_t dn[32];    //   and length
  uint8_t par[32];    // entry index in the previous level
  uint8_t dsel[32];   // back entry that is the driver
  uint32_t cnt, cur_e, cur_k, pad;
};

size_t search_smem_bytes(uint32_t n_q, uint32_t warps) {
  const uint32_t levels = n_q > 2 ? n_q - 2 : 1;
  return (size_t)warps * levels * sizeof(LevelSM);
}

__device__ __forceinline__ bool d2_bit(const uint64_t* d2, uint64_t words, uint32_t q, uint32_t v) {
  return (d2[(uint64_t)q * words + (v >> 6)] >> (v & 63)) & 1ULL;
}

__global__ void k_seed(uint32_t B, const UpdInfo* info, DevGraph g, const Plan* plan, const uint64_t* d2,
                       uint64_t d2_words, Task* tasks, unsigned int* n_tasks, uint32_t task_cap,
                       uint32_t* safe, unsigned int* error, uint32_t shard_rank, uint32_t shard_count,
                       uint32_t turboflux_compat, uint32_t dup_zero) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  const UpdInfo u = info[s];
  uint32_t sf = 1;
  // dup_zero: an insertion of a present edge counts nothing (CaLiG skips it,
  // ParaCOSM/CSM/matching/Parallel_CaLiG/parallel_calig.cpp:1249)
  if ((u.flags & UF_VALID) && !(u.flags & UF_INVALID) && !(dup_zero && (u.flags & UF_DUP))) {
    const uint32_t L1 = g.vlabel[u.v1], L2 = g.vlabel[u.v2], l = u.label;
    const uint32_t na = plan->n_anchor;
    // The reference's TurboFlux deletion seeds every query edge whose vertex
    // labels match, whatever its edge label, and filters the endpoints by d2
    // only on spanning-tree edges (ParaCOSM/CSM/matching/TurboFlux/turboflux.cpp:966-1022)
    const bool compat_del = turboflux_compat && !(u.flags & UF_ADD);
    for (uint32_t a = 0; a < na; a++) {
      const PlanAnchor* A = &plan->anchors[a];
      if (A->el != l && !compat_del) continue;
      const bool o0 = A->la == L1 && A->lb == L2;
      const bool o1 = A->la == L2 && A->lb == L1;
      if (!(o0 || o1)) continue;
      sf = 0;
      for (int o = 0; o < 2; o++) {
        if (!(o ? o1 : o0)) continue;
        const uint32_t x = o ? u.v2 : u.v1, y = o ? u.v1 : u.v2;
        if (d2 && (!compat_del || A->tree) &&
            !(d2_bit(d2, d2_words, A->pos[0].qv, x) && d2_bit(d2, d2_words, A->pos[1].qv, y)))
          continue;
        if (shard_count > 1 && (s + 2 * a + (uint32_t)o) % shard_count != shard_rank) continue;  // another GPU's
        unsigned int i = atomicAdd(n_tasks, 1u);
        if (i >= task_cap) { atomicExch(error, kErrTaskOverflow); continue; }
        tasks[i] = Task{s, (uint16_t)a, (uint8_t)o, 0};
      }
    }
  }
  safe[s] = sf;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= (uint32_t)o) v += t;
  }
  return v;
}

// Bounds of up to four back segments of one position for one prefix, with
// the batch touch count of each row (0: the row holds no entry inserted or
// deleted in this batch, so every entry of it is present at every batch time).
struct SegQuad {
  uint32_t v[4], c[4], lo[4], hi[4], tc[4];
};

// Loads back entries b0 .. b0 + 3 of position P for prefix m: all loads are
// independent, so the quad costs one round trip to L2.  The bounds of entry
// `skip` are not loaded (the driver: the candidate came from it), but its
// touch count is (its edge still needs the batch-time presence test).
__device__ __forceinline__ void load_quad(const DevGraph& g, const PlanAnchor* A, const PlanPos& P, uint32_t b0,
                                          const uint32_t* m, uint32_t skip, SegQuad& s) {
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const uint32_t b = b0 + (uint32_t)i;
    s.v[i] = 0; s.c[i] = 0; s.lo[i] = 0; s.hi[i] = 0; s.tc[i] = 0;
    if (b < P.nb) {
      s.v[i] = m[A->back_pos[P.boff + b]];
      s.c[i] = A->back_combo[P.boff + b];
      if (b != skip) {
        const uint32_t* d = g.dir + (size_t)s.v[i] * (g.nc + 1) + s.c[i];
        const uint32_t base = (uint32_t)g.row_off[s.v[i]];
        s.lo[i] = base + d[0];
        s.hi[i] = base + d[1];
      }
      s.tc[i] = g.t_count[s.v[i]];
    }
  }
}

// Is x in each loaded segment of the quad (every entry but `skip`), and is
// every back edge of the quad present at batch time t?  The lower-bound
// searches of the four segments advance in lockstep (one round trip per
// round); a probe that lands on x ends that search, so no separate load
// confirms the final position (if x is in the segment, the search must probe
// its slot before it can end there).
__device__ __forceinline__ bool quad_joins(const DevGraph& g, const uint32_t* pool, const PlanPos& P, uint32_t b0,
                                           uint32_t skip, uint32_t x, int32_t t, SegQuad& s) {
  uint32_t need = 0, found = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const uint32_t b = b0 + (uint32_t)i;
    if (b < P.nb && b != skip) need |= 1u << i;
  }
  for (;;) {
    bool more = false;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      if (s.lo[i] < s.hi[i]) {
        const uint32_t mid = (s.lo[i] + s.hi[i]) >> 1;
        const uint32_t val = pool[mid];
        if (val < x) s.lo[i] = mid + 1;
        else if (val > x) s.hi[i] = mid;
        else { found |= 1u << i; s.hi[i] = s.lo[i]; }
        more = true;
      }
    }
    if (!more) break;
  }
  if ((found & need) != need) return false;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    if (b0 + (uint32_t)i >= P.nb || s.tc[i] == 0) continue;
    if (!present_at(g, s.v[i], s.c[i], x, t)) return false;
  }
  return true;
}

// Full candidate check of data vertex x for position `pos` given the matched
// prefix m[0 .. pos-1]; `dsel` is the back entry whose segment produced x and
// q0 the first quad of pos's back entries, already loaded (load_quad with
// skip = dsel).  The candidate-filter word is loaded before the first join
// round and tested after it, so the two round trips overlap.
__device__ __forceinline__ bool check_candidate_q(const SearchParams& p, const uint32_t* pool, const PlanAnchor* A,
                                                  uint32_t pos, uint32_t x, const uint32_t* m, uint32_t dsel,
                                                  int32_t t, SegQuad& q0, uint32_t lab_mask = 0xffffffffu) {
  const PlanPos P = A->pos[pos];
  const uint64_t fw = p.d2 ? p.d2[(uint64_t)P.qv * p.d2_words + (x >> 6)] : ~0ULL;
  bool ok = true;
  if (!p.homo) {
    for (uint32_t mk = P.samelab & lab_mask; mk; mk &= mk - 1) ok &= m[__ffs(mk) - 1] != x;
  }
  if (!ok) return false;
  ok = quad_joins(p.g, pool, P, 0, dsel, x, t, q0);
  if (!((fw >> (x & 63)) & 1ULL)) return false;
  if (!ok) return false;
  for (uint32_t b0 = 4; b0 < P.nb; b0 += 4) {
    SegQuad q;
    load_quad(p.g, A, P, b0, m, dsel, q);
    if (!quad_joins(p.g, pool, P, b0, dsel, x, t, q)) return false;
  }
  return true;
}

// The same check with the edge table (DevGraph::ekeys): each join is one
// probe for the key of edge (m[b], x) with back entry b's edge label.  The
// candidate-filter word comes first (the filter is small and stays in L2),
// then the joins one at a time, stopping at the first that fails: the table
// is larger than L2, every probe of it is a random line fetched from HBM, and
// HBM is what bounds this search -- most candidates fail their first join,
// and probing all back entries at once (four in flight) fetched three times
// the lines for a candidate that one probe settles.  The batch-time presence
// of the back edges is tested for the candidates that pass.
__device__ __forceinline__ bool check_candidate_h(const SearchParams& p, const PlanAnchor* A, uint32_t pos,
                                                  uint32_t x, const uint32_t* m, uint32_t dsel, int32_t t,
                                                  uint32_t lab_mask = 0xffffffffu) {
  const PlanPos P = A->pos[pos];
  const DevGraph& g = p.g;
  const uint64_t fw = p.d2 ? ld_stream(p.d2 + (uint64_t)P.qv * p.d2_words + (x >> 6)) : ~0ULL;
  bool ok = true;
  if (!p.homo) {
    for (uint32_t mk = P.samelab & lab_mask; mk; mk &= mk - 1) ok &= m[__ffs(mk) - 1] != x;
  }
  if (!ok) return false;
  if (!((fw >> (x & 63)) & 1ULL)) return false;
  for (uint32_t b = 0; b < P.nb; b++) {
    if (b == dsel) continue;
    const uint64_t key = edge_key(m[A->back_pos[P.boff + b]], x, A->back_combo[P.boff + b] % g.n_el);
    const uint64_t slot = edge_slot(key, g.emask);
    if (!edge_probe_rest(g, key, slot, ld_stream(g.ekeys + slot))) return false;
  }
  for (uint32_t b = 0; b < P.nb; b++) {
    const uint32_t v = m[A->back_pos[P.boff + b]];
    if (g.t_count[v] && !present_at(g, v, A->back_combo[P.boff + b], x, t)) return false;
  }
  return true;
}

// The same check when no quad was prefetched.
__device__ __forceinline__ bool check_candidate(const SearchParams& p, const uint32_t* pool, const PlanAnchor* A,
                                                uint32_t pos, uint32_t x, const uint32_t* m, uint32_t dsel,
                                                int32_t t, uint32_t lab_mask = 0xffffffffu) {
  if (p.g.emask) return check_candidate_h(p, A, pos, x, m, dsel, t, lab_mask);
  SegQuad q0;
  load_quad(p.g, A, A->pos[pos], 0, m, dsel, q0);
  return check_candidate_q(p, pool, A, pos, x, m, dsel, t, q0, lab_mask);
}

// Number of entries of segment (v, c) = [lo, hi) present at batch time t,
// given the row's touch count tc (seg_size_at with the count already loaded).
__device__ __forceinline__ uint32_t seg_size_tc(const DevGraph& g, uint32_t v, uint32_t c, uint32_t lo, uint32_t hi,
                                                uint32_t tc, int32_t t) {
  if (tc == 0 || hi == lo) return hi - lo;
  return seg_size_at(g, v, c, lo, hi, t);
}

// Driver segment of position np for prefix m (the smallest union-graph back
// segment); false if some back segment is empty at batch time t.  `bytes`
// receives 4 B x the sizes at time t of all back segments: the algorithmic
// bytes of expanding this node.  Segment bounds and touch counts are loaded
// four back entries at a time.
__device__ __forceinline__ bool pick_driver(const SearchParams& p, const PlanAnchor* A, uint32_t np,
                                            const uint32_t* m, int32_t t, uint32_t& dlo, uint32_t& dn,
                                            uint32_t& dsel, unsigned long long& bytes) {
  const PlanPos P = A->pos[np];
  uint32_t best = 0xffffffffu;
  bool empty = false;
  unsigned long long b4 = 0;
  for (uint32_t b0 = 0; b0 < P.nb; b0 += 4) {
    SegQuad q;
    load_quad(p.g, A, P, b0, m, 0xffffffffu, q);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const uint32_t b = b0 + (uint32_t)i;
      if (b >= P.nb) continue;
      const uint32_t sz = q.hi[i] - q.lo[i];
      const uint32_t szt = seg_size_tc(p.g, q.v[i], q.c[i], q.lo[i], q.hi[i], q.tc[i], t);
      b4 += 4ull * szt;
      if (szt == 0) empty = true;
      if (sz < best) { best = sz; dsel = b; dlo = q.lo[i]; }
    }
  }
  dn = best;
  bytes = b4;
  return !empty;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Per-task accumulators, flushed to the update's counters when the task ends.
struct TaskAcc {
  unsigned long long cnt, hash, bytes, iters, checks, checks_hungry;
};

// Hands unexpanded work at the shallowest level with work left to idle warps:
// whole entries from the end of that level's buffer, or, when only the entry
// in progress is left, the upper half of its remaining driver range.  Each
// donated task is a partial match (positions 0..L) plus a driver range for
// position L + 1.  Returns the number of tasks handed over.
__device__ uint32_t donate(const SearchParams& p, LevelSM* lv, int d, uint32_t lane, uint32_t idle_now,
                           uint32_t t, const Task& T, uint32_t m0, uint32_t m1, int tail_level) {
  // Ranges are split down to two elements near the root (where every element
  // heads a large subtree) and only from 64 elements further down.
  const int n = (int)p.plan->n;
  int Ls = 0;
  uint32_t mode = 0;  // 1: whole entries, 2: split the entry in progress
  for (int L = 1; L <= d && L <= n - 2; L++) {
    const uint32_t cnt = lv[L].cnt, ce = lv[L].cur_e;
    if (ce >= cnt) continue;
    if (cnt - ce >= 2) { Ls = L; mode = 1; break; }
    if (L == tail_level) continue;  // the tail stage takes whole entries only
    const uint32_t min_split = (L + 5 <= n) ? 2u : (p.split_deep ? p.split_deep : 64u);
    if (lv[L].dn[ce] - lv[L].cur_k >= min_split) { Ls = L; mode = 2; break; }
  }
  if (!mode) {
    if (lane == 0) atomicAdd(&p.sstat->starved, 1ULL);
    return 0;
  }
  LevelSM& S = lv[Ls];
  const uint32_t cnt = S.cnt, ce = S.cur_e;
  const uint32_t avail = mode == 1 ? min(cnt - ce - 1, 32u) : 1u;
  // take up to `avail` units of hunger (idle warps not yet promised a
  // record; a signed count): one subtraction, the excess given back, no
  // retries however many warps donate at once
  unsigned long long base = 0;
  uint32_t k = 0;
  if (lane == 0) {
    const uint32_t want = min(avail, idle_now);
    const int old = (int)atomicSub(&p.q->hungry, want);
    k = old <= 0 ? 0u : min((uint32_t)old, want);
    if (k < want) atomicAdd(&p.q->hungry, want - k);
    if (k) {
      atomicAdd(&p.q->pending, k);
      base = atomicAdd(&p.q->tail, (unsigned long long)k);
      atomicAdd(&p.sstat->donations, 1ULL);
    }
  }
  k = __shfl_sync(0xffffffffu, k, 0);
  if (k == 0) return 0;
  base = __shfl_sync(0xffffffffu, base, 0);
  // entry handed to lane j and its driver range
  uint32_t e = 0, dlo = 0, dn = 0;
  if (mode == 1) {
    e = cnt - k + lane;
    if (lane < k) { dlo = S.dlo[e]; dn = S.dn[e]; }
  } else {
    e = ce;
    const uint32_t rem = S.dn[ce] - S.cur_k, keep = rem >> 1;
    dlo = S.dlo[ce] + S.cur_k + keep;
    dn = rem - keep;
  }
  if (lane < k) {
    const unsigned long long ticket = base + lane;
    const uint32_t slot = (uint32_t)(ticket & (p.qcap - 1));
    // the slot is free for this ticket once its previous reader released it
    volatile unsigned long long* sq = p.qseq + slot;
    const unsigned long long t0 = global_ns();
    bool ok = true;
    while (*sq != ticket) {
      __nanosleep(64);
      if (global_ns() - t0 > p.slot_limit_ns) { atomicExch(p.error, kErrWaitTimeout); ok = false; break; }
    }
    DTask* D = p.dq + slot;
    uint32_t idx = e;
    for (int L = Ls; L >= 2; --L) { D->m[L] = lv[L].v[idx]; idx = lv[L].par[idx]; }
    D->m[0] = m0; D->m[1] = m1;
    D->upd = ok ? t : 0xffffffffu;  // a record that could not be placed is published as void
    D->anchor = T.anchor; D->orient = T.orient; D->depth = (uint8_t)Ls;
    D->dlo = dlo; D->dn = dn; D->dsel = S.dsel[e];
    __threadfence();
    *sq = ticket + 1;  // publish
  }
  __syncwarp();
  if (lane == 0) {
    if (mode == 1) S.cnt = cnt - k;
    else S.dn[ce] = S.cur_k + ((S.dn[ce] - S.cur_k) >> 1);
  }
  __syncwarp();
  return k;
}

// ---------------------------------------------------------------- tail stage

constexpr unsigned long long kTailSat = 1ULL << 58;  // a warp's sum of 32 saturated counts stays below 2^63

__device__ __forceinline__ unsigned long long sat_mul(unsigned long long a, unsigned long long b) {
  if (a == 0 || b == 0) return 0;
  return a > kTailSat / b ? kTailSat : min(kTailSat, a * b);
}

// Injective assignments of a label group of g <= kTailGroup tail positions,
// from N[M]: the number of candidates whose set of group members they are a
// candidate of is exactly M.  Members served by candidates of one class M
// form a subset R of M, in N[M] (N[M] - 1) ... (N[M] - |R| + 1) ways; a
// dynamic program over the set of served members.  Without injectivity
// (homo) it is the product of the members' candidate counts.  Saturates.
__device__ __noinline__ unsigned long long group_assignments(uint32_t g, const unsigned long long* N, int homo) {
  const uint32_t full = (1u << g) - 1u;
  if (homo) {
    unsigned long long prod = 1;
    for (uint32_t i = 0; i < g; i++) {
      unsigned long long c = 0;
      for (uint32_t M = 1; M <= full; M++)
        if ((M >> i) & 1u) c = min(kTailSat, c + N[M]);
      prod = sat_mul(prod, c);
    }
    return prod;
  }
  unsigned long long f[1u << kTailGroup], h[1u << kTailGroup];
  for (uint32_t S = 0; S <= full; S++) f[S] = S == 0 ? 1ull : 0ull;
  for (uint32_t M = 1; M <= full; M++) {
    if (!N[M]) continue;
    for (uint32_t S = 0; S <= full; S++) h[S] = 0;
    for (uint32_t S = 0; S <= full; S++) {
      if (!f[S]) continue;
      const uint32_t fr = M & ~S;
      for (uint32_t R = fr;; R = (R - 1u) & fr) {  // every subset of fr, the empty one last
        unsigned long long ways = 1;
        for (uint32_t r = 0, k = (uint32_t)__popc(R); r < k; r++) ways = sat_mul(ways, N[M] > r ? N[M] - r : 0ull);
        if (ways) h[S | R] = min(kTailSat, h[S | R] + sat_mul(f[S], ways));
        if (R == 0) break;
      }
    }
    for (uint32_t S = 0; S <= full; S++) f[S] = h[S];
  }
  return f[full];
}

// Prefix m[0 .. L] of entry e of level L.
__device__ __forceinline__ void load_prefix(uint32_t* m, const LevelSM* lv, int L, uint32_t e, uint32_t m0,
                                            uint32_t m1) {
  m[0] = m0; m[1] = m1;
  uint32_t idx = e;
  for (int l2 = L; l2 >= 2; --l2) { m[l2] = lv[l2].v[idx]; idx = lv[l2].par[idx]; }
}

// Counts the completions of the entries of level L (= the anchor's tail_at:
// complete matches of the positions before the independent tail).  For each
// label group of the tail, every member's candidates are listed from its
// driver segment (32 (entry, element) pairs at a time, as in run_levels) and
// classified by the other members they are candidates of; a candidate is
// counted under the first member it belongs to, in per-entry class counters
// kept in the unused levels above L.  Each entry's completions are the
// product over groups of group_assignments.  A group is not looked at for
// entries whose product is already 0.  Returns false when the update was
// stopped (cap, deadline or stop flag).
__device__ __forceinline__ bool tail_stage(const SearchParams& p, const uint32_t* pool, LevelSM* lv, int L,
                                        uint32_t lane, const Task& T, const PlanAnchor* A, uint32_t m0,
                                        uint32_t m1, TaskAcc& acc) {
  const uint32_t t = T.upd;
  volatile unsigned int* stop = p.stop;
  LevelSM& S = lv[L];
  const uint32_t ce = S.cur_e, cnt = S.cnt, ck = S.cur_k;
  const uint32_t ne = cnt > ce ? cnt - ce : 0u;
  const bool has = lane < ne;
  const uint32_t e_mine = ce + (has ? lane : 0u);
  uint32_t* cntr = reinterpret_cast<uint32_t*>(&lv[L + 1]);  // [class][entry], levels L+1.. are unused here
  const uint32_t pmask = A->prefix_mask;
  uint32_t m[kMaxQ];
  unsigned long long prod = has ? 1ull : 0ull, bytes = 0;
  bool stopped = false;
  uint32_t gp = 0, it = 0;
  for (uint32_t gi = 0; gi < A->n_groups; gi++) {
    const uint32_t g = A->gsize[gi];
    const uint32_t ncls = (1u << g) - 1u;
    for (uint32_t c = 0; c < ncls; c++) cntr[c * 32 + lane] = 0;
    __syncwarp();
    for (uint32_t j = 0; j < g && !stopped; j++) {
      const uint32_t ps = A->gpos[gp + j];
      uint32_t dlo = 0, dn = 0, dsel = 0;
      if (prod) {
        if (ps == (uint32_t)L + 1) {  // the entry's own driver, found when it was pushed
          const uint32_t skip = lane == 0 ? ck : 0u;
          dlo = S.dlo[e_mine] + skip; dn = S.dn[e_mine] - skip; dsel = S.dsel[e_mine];
        } else {
          load_prefix(m, lv, L, e_mine, m0, m1);
          unsigned long long b4 = 0;
          if (!pick_driver(p, A, ps, m, (int32_t)t, dlo, dn, dsel, b4)) dn = 0;
          bytes += b4;
        }
      }
      const uint32_t incl = warp_incl_scan(dn, lane);
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
      for (uint32_t base = 0; base < total; base += 32) {
        if ((++it & 63) == 0) {
          unsigned int st = 0;
          if (lane == 0) {
            if (p.deadline_ns && global_ns() - p.sstat->launch_t0 > p.deadline_ns)
              atomicCAS(const_cast<unsigned int*>(stop) + t, 0u, kStopDeadline);
            st = stop[t];
          }
          if (__shfl_sync(0xffffffffu, st, 0)) { stopped = true; break; }
        }
        acc.iters++;
        const uint32_t gidx = base + lane;
        uint32_t owner = 0;
#pragma unroll
        for (uint32_t step = 16; step; step >>= 1) {
          const uint32_t v = __shfl_sync(0xffffffffu, incl, owner + step - 1);
          if (v <= gidx) owner += step;
        }
        const uint32_t own = owner & 31u;
        const uint32_t prev = __shfl_sync(0xffffffffu, incl, (owner - 1u) & 31u);
        const uint32_t o_dlo = __shfl_sync(0xffffffffu, dlo, own);
        const uint32_t o_dsel = __shfl_sync(0xffffffffu, dsel, own);
        if (gidx < total) {
          const uint32_t kk = gidx - (owner ? prev : 0u);
          const uint32_t x = ld_stream(pool + (uint64_t)o_dlo + kk);
          load_prefix(m, lv, L, ce + owner, m0, m1);
          if (check_candidate(p, pool, A, ps, x, m, o_dsel, (int32_t)t, pmask)) {
            uint32_t M = 1u << j;
            bool seen = false;
            for (uint32_t i = 0; i < g && !seen; i++) {
              if (i == j || !check_candidate(p, pool, A, A->gpos[gp + i], x, m, 0xffu, (int32_t)t, pmask)) continue;
              if (i < j) seen = true;
              else M |= 1u << i;
            }
            if (!seen) atomicAdd(&cntr[(M - 1u) * 32u + owner], 1u);
          }
        }
      }
      __syncwarp();
    }
    gp += g;
    if (stopped) break;
    if (prod) {
      unsigned long long N[1u << kTailGroup];
      N[0] = 0;
      for (uint32_t c = 1; c <= ncls; c++) N[c] = cntr[(c - 1u) * 32u + lane];
      prod = sat_mul(prod, group_assignments(g, N, p.homo));
    }
    __syncwarp();
    if (!__any_sync(0xffffffffu, prod != 0)) break;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
  acc.bytes += bytes;
  if (stopped) return false;
  unsigned long long sum = prod;
#pragma unroll
  for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if (lane == 0) S.cur_e = cnt;
  __syncwarp();
  acc.cnt += sum;
  if (sum && p.cap) {
    unsigned int hit = 0;
    if (lane == 0) {
      const unsigned long long old = atomicAdd(&p.count[t], acc.cnt);
      acc.cnt = 0;
      if (old + sum >= p.cap) { stop[t] = kStopCap; hit = 1; }
    }
    if (__shfl_sync(0xffffffffu, hit, 0)) return false;
  }
  return true;
}

// Depth-first walk over chunked levels starting at level `d` (see the file
// comment); positions 0 and 1 hold m0 and m1.  MODE 1 compiles the
// match-set append in, MODE 2 the tail stage; each is a separate
// instantiation so that the plain counting kernel (MODE 0) keeps its
// register budget.
template <int MODE>
__device__ void run_levels(const SearchParams& p, const uint32_t* pool, LevelSM* lv, int d, uint32_t lane,
                           const Task& T, const PlanAnchor* A, uint32_t m0, uint32_t m1, TaskAcc& acc) {
  const uint32_t n = p.plan->n;
  const uint32_t t = T.upd;
  volatile unsigned int* stop = p.stop;
  uint32_t iter = 0;
  const unsigned long long t_start = global_ns();
  constexpr bool EN = MODE == 1;
  const int tail_level = (MODE == 2 && p.tail && A->tail_at) ? (int)A->tail_at : -1;
  uint32_t seen_stop = 0, seen_hungry = 0;  // lane 0: flags loaded in the previous iteration
  while (d >= 1) {
    ++iter;
    if ((iter & 63) == 0 && p.deadline_ns) {
      unsigned int late = 0;
      if (lane == 0 && global_ns() - p.sstat->launch_t0 > p.deadline_ns) {
        atomicCAS(const_cast<unsigned int*>(stop) + t, 0u, kStopDeadline);
        late = 1;
      }
      if (__shfl_sync(0xffffffffu, late, 0)) break;
    }
    if ((iter & 63) == 0) {
      unsigned int expired = (lane == 0) ? (global_ns() - t_start > p.task_limit_ns) : 0u;
      if (__shfl_sync(0xffffffffu, expired, 0)) {
        if (lane == 0) {
          atomicExch(p.error, kErrTaskGuard);
          if (atomicCAS(&p.sstat->guard_set, 0u, 1u) == 0u) {
            p.sstat->guard_d = (unsigned)d; p.sstat->guard_upd = t; p.sstat->guard_iters = iter;
            for (int L = 1; L <= d && L <= 16; L++) {
              const uint32_t ce = lv[L].cur_e;
              p.sstat->guard_lv[4 * (L - 1) + 0] = lv[L].cnt;
              p.sstat->guard_lv[4 * (L - 1) + 1] = ce;
              p.sstat->guard_lv[4 * (L - 1) + 2] = lv[L].cur_k;
              p.sstat->guard_lv[4 * (L - 1) + 3] = ce < 32 ? lv[L].dn[ce] : 0xffffffffu;
            }
          }
        }
        break;
      }
    }
    if ((iter & 7) == 0) {
      if (__shfl_sync(0xffffffffu, seen_stop, 0)) break;
    }
    if ((iter & (p.donate_every ? p.donate_every - 1 : 0u)) == 0 && p.dq) {
      const uint32_t idle_now = __shfl_sync(0xffffffffu, seen_hungry, 0);
      acc.checks++;
      if (idle_now) acc.checks_hungry++;
      if (idle_now) donate(p, lv, d, lane, idle_now, t, T, m0, m1, tail_level);
    }
    // the stop flag and the idle-warp count the checks above read are loaded
    // one iteration ahead, so their round trip to L2 overlaps a step's work
    // instead of preceding it (a step late is soon enough for both), and only
    // before the iterations that read them: each load is a round trip to a
    // line other warps update
    if (lane == 0 && (iter & 3) == 3) {
      seen_stop = stop[t];
      seen_hungry = p.dq ? (uint32_t)max((int)*(volatile unsigned int*)&p.q->hungry, 0) : 0u;
    }
    if constexpr (MODE == 2) {
      if (d == tail_level) {
        if (!tail_stage(p, pool, lv, d, lane, T, A, m0, m1, acc)) break;
        d--;
        continue;
      }
    }
    LevelSM& L = lv[d];
    const uint32_t cnt = L.cnt, ce = L.cur_e, ck = L.cur_k;
    if (ce >= cnt) { d--; continue; }
    acc.iters++;
    // the next 32 (entry, driver element) pairs of this level
    const uint32_t el = ce + lane;
    const uint32_t rem = (el < cnt) ? L.dn[el] - (lane == 0 ? ck : 0u) : 0u;
    const uint32_t incl = warp_incl_scan(rem, lane);
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t owner = 0;
#pragma unroll
    for (uint32_t step = 16; step; step >>= 1) {
      const uint32_t v = __shfl_sync(0xffffffffu, incl, owner + step - 1);
      if (v <= lane) owner += step;
    }
    const uint32_t prev = __shfl_sync(0xffffffffu, incl, owner > 0 ? (owner - 1) & 31 : 0);
    const bool active = lane < total;
    const uint32_t e = ce + owner;
    const uint32_t kk = lane - (owner > 0 ? prev : 0u) + (owner == 0 ? ck : 0u);
    uint32_t nce, nck;
    if (total <= 32) {
      nce = ce + min(32u, cnt - ce); nck = 0;
    } else {
      const uint32_t o31 = __shfl_sync(0xffffffffu, owner, 31);
      const uint32_t k31 = __shfl_sync(0xffffffffu, kk, 31);
      const uint32_t e31 = ce + o31;
      if (k31 + 1 >= L.dn[e31]) { nce = e31 + 1; nck = 0; } else { nce = e31; nck = k31 + 1; }
    }
    const uint32_t pos = (uint32_t)d + 1;
    bool valid = false;
    uint32_t x = 0, ndlo = 0, ndn = 0, ndsel = 0;
    unsigned long long nb4 = 0;
    uint32_t m[kMaxQ];
    bool act = active;
    if (act && (e >= cnt || kk >= L.dn[e])) {  // lanes disagree on the level state: flag it, read nothing
      atomicExch(p.error, kErrBadTask);
      act = false;
    }
    if (act) {
      // the candidate and the first back segments of its position are loaded
      // together: the segments depend on the prefix only
      x = ld_stream(pool + (uint64_t)L.dlo[e] + kk);
      m[0] = m0; m[1] = m1;
      uint32_t idx = e;
      for (int l2 = d; l2 >= 2; --l2) { m[l2] = lv[l2].v[idx]; idx = lv[l2].par[idx]; }
      const uint32_t ds = L.dsel[e];
      if (p.g.emask) {
        valid = check_candidate_h(p, A, pos, x, m, ds, (int32_t)t);
      } else {
        SegQuad q0;
        load_quad(p.g, A, A->pos[pos], 0, m, ds, q0);
        valid = check_candidate_q(p, pool, A, pos, x, m, ds, (int32_t)t, q0);
      }
      if (valid && pos + 1 < n) {
        m[pos] = x;
        valid = pick_driver(p, A, pos + 1, m, (int32_t)t, ndlo, ndn, ndsel, nb4);
      }
    }
    __syncwarp();
    if (lane == 0) { L.cur_e = nce; L.cur_k = nck; }
    __syncwarp();  // the cursor must be visible to every lane before the next iteration reads it
    const uint32_t mask = __ballot_sync(0xffffffffu, valid);
    if (pos + 1 < n) {
#pragma unroll
      for (int o = 16; o; o >>= 1) nb4 += __shfl_xor_sync(0xffffffffu, nb4, o);
      acc.bytes += nb4;
    }
    if (pos == n - 1) {
      const uint32_t c = __popc(mask);
      if (EN) {
        unsigned long long base = 0;
        if (lane == 0 && c) base = atomicAdd(p.enum_n, (unsigned long long)c);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (valid) {
          const unsigned long long r = base + __popc(mask & ((1u << lane) - 1u));
          if (r < p.enum_cap) {
            uint32_t* rec = p.enum_buf + r * p.enum_stride;
            rec[0] = p.enum_base + t;
            rec[1 + A->pos[pos].qv] = x;
            for (uint32_t q = 0; q < pos; q++) rec[1 + A->pos[q].qv] = m[q];
          }
        }
      }
      if (p.want_hash) {
        unsigned long long h = 0;
        if (valid) {
          uint64_t s = pair_hash(A->pos[pos].qv, x);
          for (uint32_t q = 0; q < pos; q++) s += pair_hash(A->pos[q].qv, m[q]);
          h = mix64(s);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
        acc.hash += h;
      }
      acc.cnt += c;
      if (c && p.cap) {
        unsigned int hit = 0;
        if (lane == 0) {
          const unsigned long long old = atomicAdd(&p.count[t], acc.cnt);
          acc.cnt = 0;
          if (old + c >= p.cap) { stop[t] = kStopCap; hit = 1; }
        }
        if (__shfl_sync(0xffffffffu, hit, 0)) break;
      }
    } else {
      LevelSM& N = lv[pos];
      if (valid) {
        const uint32_t slot = __popc(mask & ((1u << lane) - 1u));
        N.v[slot] = x; N.par[slot] = (uint8_t)e; N.dlo[slot] = ndlo; N.dn[slot] = ndn;
        N.dsel[slot] = (uint8_t)ndsel;
      }
      if (lane == 0) { N.cnt = __popc(mask); N.cur_e = 0; N.cur_k = 0; }
      __syncwarp();
      if (mask) d = (int)pos;
    }
  }
}

__device__ __forceinline__ void flush_acc(const SearchParams& p, uint32_t t, uint32_t lane, TaskAcc& acc) {
  if (lane == 0) {
    if (acc.cnt) {
      const unsigned long long old = atomicAdd(&p.count[t], acc.cnt);
      if (p.cap && old + acc.cnt >= p.cap) p.stop[t] = kStopCap;
    }
    if (p.want_hash && acc.hash) atomicAdd(&p.hash[t], acc.hash);
    if (acc.bytes) atomicAdd(&p.bytes[t], acc.bytes);
  }
  acc.cnt = 0; acc.hash = 0; acc.bytes = 0;
  __syncwarp();
}

// Root task: positions 0 and 1 are the updated edge; level 1 holds the driver
// segment of position 2.
template <int MODE>
__device__ void run_root(const SearchParams& p, const uint32_t* pool, LevelSM* lv, uint32_t lane, const Task& T,
                         TaskAcc& acc) {
  const uint32_t n = p.plan->n;
  const uint32_t t = T.upd;
  const PlanAnchor* A = &p.plan->anchors[T.anchor];
  const UpdInfo U = p.info[t];
  const uint32_t m0 = T.orient ? U.v2 : U.v1, m1 = T.orient ? U.v1 : U.v2;
  if (n == 2) {
    if (lane == 0) {
      acc.cnt += 1;
      if (p.want_hash) acc.hash += mix64(pair_hash(A->pos[0].qv, m0) + pair_hash(A->pos[1].qv, m1));
      if (MODE == 1) {
        const unsigned long long r = atomicAdd(p.enum_n, 1ull);
        if (r < p.enum_cap) {
          uint32_t* rec = p.enum_buf + r * p.enum_stride;
          rec[0] = p.enum_base + t;
          rec[1 + A->pos[0].qv] = m0;
          rec[1 + A->pos[1].qv] = m1;
        }
      }
    }
    return;
  }
  const PlanPos P2 = A->pos[2];
  uint32_t sz = 0xffffffffu, szt = 1;
  uint64_t lo = 0, hi = 0;
  unsigned long long rb = 0;
  if (lane < P2.nb) {
    const uint32_t j = A->back_pos[P2.boff + lane], c = A->back_combo[P2.boff + lane];
    const uint32_t v = j == 0 ? m0 : m1;
    segment(p.g, v, c, lo, hi);
    sz = (uint32_t)(hi - lo);
    szt = seg_size_at(p.g, v, c, lo, hi, (int32_t)t);
    rb = 4ull * szt;
  }
  const bool root_empty = __any_sync(0xffffffffu, szt == 0);
#pragma unroll
  for (int o = 16; o; o >>= 1) rb += __shfl_xor_sync(0xffffffffu, rb, o);
  acc.bytes += rb;
  uint64_t key = ((uint64_t)sz << 32) | lane;
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    uint64_t other = __shfl_xor_sync(0xffffffffu, key, o);
    key = other < key ? other : key;
  }
  const uint32_t minsz = root_empty ? 0u : (uint32_t)(key >> 32), sel = (uint32_t)key;
  const uint32_t dlo0 = (uint32_t)__shfl_sync(0xffffffffu, lo, sel);
  if (minsz == 0) return;
  if (lane == 0) {
    lv[1].cnt = 1; lv[1].cur_e = 0; lv[1].cur_k = 0;
    lv[1].dlo[0] = dlo0; lv[1].dn[0] = minsz; lv[1].dsel[0] = (uint8_t)sel;
  }
  __syncwarp();
  run_levels<MODE>(p, pool, lv, 1, lane, T, A, m0, m1, acc);
}

// Donated task: rebuild the chain of the partial match (exhausted levels
// 1 .. depth-1) and continue from level `depth`.  `hw` holds record words
// 0..4 in lanes 0..4 and `mv` holds m[lane] (see DTask).
template <int MODE>
__device__ void run_donated(const SearchParams& p, const uint32_t* pool, LevelSM* lv, uint32_t lane, uint32_t hw,
                            uint32_t mv, TaskAcc& acc, uint32_t& upd_out, unsigned long long ticket,
                            unsigned long long seen_seq) {
  const uint32_t upd = __shfl_sync(0xffffffffu, hw, 0);
  const uint32_t w1 = __shfl_sync(0xffffffffu, hw, 1);
  const uint32_t dlo = __shfl_sync(0xffffffffu, hw, 2);
  const uint32_t dn = __shfl_sync(0xffffffffu, hw, 3);
  const uint32_t dsel = __shfl_sync(0xffffffffu, hw, 4);
  const uint32_t anchor = w1 & 0xffffu, orient = (w1 >> 16) & 0xffu, depth = w1 >> 24;
  const uint32_t n = p.plan->n;
  upd_out = upd;
  if (upd == 0xffffffffu) return;  // void record (its donor flagged an error)
  if (upd >= p.batch || anchor >= p.plan->n_anchor || depth < 1 || depth + 2 > n || dn == 0 ||
      (unsigned long long)dlo + dn > p.g.pool_cap) {
    if (lane == 0) {
      atomicExch(p.error, kErrBadTask);
      if (atomicCAS(&p.sstat->bad_set, 0u, 1u) == 0u) {
        p.sstat->bad_ticket = ticket; p.sstat->bad_seq = seen_seq; p.sstat->bad_batch = p.batch;
        p.sstat->bad_words[0] = upd; p.sstat->bad_words[1] = w1; p.sstat->bad_words[2] = dlo;
        p.sstat->bad_words[3] = dn; p.sstat->bad_words[4] = dsel;
      }
    }
    upd_out = 0xffffffffu;
    return;
  }
  Task T{upd, (uint16_t)anchor, (uint8_t)orient, 0};
  const PlanAnchor* A = &p.plan->anchors[anchor];
  const uint32_t m0 = __shfl_sync(0xffffffffu, mv, 0), m1 = __shfl_sync(0xffffffffu, mv, 1);
  for (uint32_t L = 1; L <= depth; L++) {
    const uint32_t v = __shfl_sync(0xffffffffu, mv, L);
    if (lane == 0) {
      LevelSM& S = lv[L];
      S.cnt = 1; S.cur_k = 0; S.v[0] = v; S.par[0] = 0;
      S.cur_e = (L < depth) ? 1u : 0u;
      if (L == depth) { S.dlo[0] = dlo; S.dn[0] = dn; S.dsel[0] = (uint8_t)dsel; }
    }
  }
  __syncwarp();
  const unsigned int stopped =
      __shfl_sync(0xffffffffu, lane == 0 ? *(volatile unsigned int*)(p.stop + upd) : 0u, 0);
  if (stopped) return;
  run_levels<MODE>(p, pool, lv, (int)depth, lane, T, A, m0, m1, acc);
}

// Per launch: tickets keep counting up across launches (the ring's slot
// sequence numbers stay consistent); hunger and pending start afresh, and the
// tickets that warps still waiting at the end of the last launch held (never
// filled) are handed out again.
__global__ void k_search_prep(SearchQueue* q, const unsigned int* n_tasks, uint32_t task_cap, SearchStats* ss,
                              unsigned int* error) {
  if (q->head < q->tail) atomicExch(error, kErrRingState);
  q->head = q->tail;  // tickets that waiting warps held when the last launch ended were never filled
  q->hungry = 0;
  q->pending = min(*n_tasks, task_cap);
  ss->launch_t0 = global_ns();
}

// Kernel body; MODE 0 counts (and hashes), 1 also appends match sets, 2
// counts independent tails (tail_stage).
template <int W, int MODE>
__device__ __forceinline__ void search_body(const SearchParams& p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint4 task_scratch[W * 10];  // one 160-byte record per warp
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t n = p.plan->n;
  const uint32_t nlev = n > 2 ? n - 2 : 1;
  LevelSM* lv = reinterpret_cast<LevelSM*>(smem_raw) + (size_t)warp * nlev - 1;  // levels 1 .. n-2
  const uint32_t* pool = p.g.pools[p.g.ps->active];
  const uint32_t ntask = min(*p.n_tasks, p.task_cap);
  volatile unsigned int* stop = p.stop;
  TaskAcc acc{0, 0, 0, 0, 0, 0};
  unsigned long long root_ns = 0, last_root = 0, max_task = 0;
  unsigned long long busy_ns = 0, idle_ns = 0;

  // 1. root tasks, in claim order
  for (;;) {
    uint32_t ti = 0;
    if (lane == 0) ti = atomicAdd(p.task_next, 1u);
    ti = __shfl_sync(0xffffffffu, ti, 0);
    if (ti >= ntask) break;
    const Task T = p.tasks[ti];
    const unsigned long long tb = global_ns();
    if (lane == 0 && p.deadline_ns && tb - p.sstat->launch_t0 > p.deadline_ns)
      atomicCAS(const_cast<unsigned int*>(stop) + T.upd, 0u, kStopDeadline);
    // stop flags change under our feet: one lane reads, the warp follows it
    const unsigned int stopped = __shfl_sync(0xffffffffu, lane == 0 ? stop[T.upd] : 0u, 0);
    if (!stopped) run_root<MODE>(p, pool, lv, lane, T, acc);
    const unsigned long long te = global_ns();
    busy_ns += te - tb;
    root_ns += te - tb;
    last_root = te;
    max_task = max(max_task, te - tb);
    flush_acc(p, T.upd, lane, acc);
    if (lane == 0 && p.dq) atomicSub(&p.q->pending, 1u);
  }
  if (lane == 0) {
    atomicAdd(&p.sstat->root_busy_ns, root_ns);
    if (last_root) atomicMax(&p.sstat->last_root_ns, last_root - p.sstat->launch_t0);
  }
  if (!p.dq) {
    if (lane == 0) { atomicAdd(&p.sstat->busy_ns, busy_ns); atomicAdd(&p.sstat->iters, acc.iters); }
    return;
  }
  // 2. donated tasks until every task is done.  The queue is a bounded ring
  // of DTask slots with per-slot sequence numbers: slot (ticket % qcap) holds
  // ticket T's record once seq == T + 1, and is free for ticket T + qcap once
  // its reader stores seq = T + qcap.  Claims take a ticket by fetch-and-add:
  // a compare-and-swap on the head, retried by thousands of idle warps at
  // once, took most of the warps' time late in a batch.
  volatile SearchQueue* q = p.q;
  for (;;) {
    unsigned long long claimed = ~0ULL, seen = 0;
    if (lane == 0) {
      const unsigned long long t0 = global_ns();
      // this warp's ticket, and one unit of hunger for it: donors fill the
      // tickets in order, one per unit they take
      const unsigned long long tk = atomicAdd((unsigned long long*)&p.q->head, 1ull);
      atomicAdd(&p.q->hungry, 1u);
      unsigned int nap = 32;
      for (;;) {
        const unsigned long long sv = *(volatile unsigned long long*)(p.qseq + (tk & (p.qcap - 1)));
        if (sv == tk + 1) { claimed = tk; seen = sv; break; }
        if (q->pending == 0) break;
        __nanosleep(nap);
        nap = min(nap * 2, 1024u);
        if (global_ns() - t0 > p.wait_limit_ns) { atomicExch(p.error, kErrWaitTimeout); break; }
      }
      idle_ns += global_ns() - t0;
    }
    claimed = __shfl_sync(0xffffffffu, claimed, 0);
    if (claimed == ~0ULL) break;
    // lane 0 copies the record through L2 (records share cache lines with other
    // slots) into the warp's scratch, and only then frees the slot for reuse
    uint4* scratch = task_scratch + warp * 10;
    if (lane == 0) {
      __threadfence();
      const uint32_t slot = (uint32_t)(claimed & (p.qcap - 1));
      const uint4* src = reinterpret_cast<const uint4*>(p.dq + slot);
#pragma unroll
      for (int i = 0; i < 10; i++) scratch[i] = __ldcg(src + i);
      __threadfence();
      *(volatile unsigned long long*)(p.qseq + slot) = claimed + p.qcap;
    }
    __syncwarp();
    const uint32_t* Dw = reinterpret_cast<const uint32_t*>(scratch);
    const uint32_t hw = lane < 5 ? Dw[lane] : 0u;
    const uint32_t mv = Dw[5 + lane];
    __syncwarp();
    uint32_t t = 0;
    const unsigned long long tb = global_ns();
    run_donated<MODE>(p, pool, lv, lane, hw, mv, acc, t, claimed, seen);
    busy_ns += global_ns() - tb;
    max_task = max(max_task, global_ns() - tb);
    if (t < p.batch) flush_acc(p, t, lane, acc);
    if (lane == 0) atomicSub(&p.q->pending, 1u);
  }
  if (lane == 0) {
    atomicAdd(&p.sstat->busy_ns, busy_ns);
    atomicAdd(&p.sstat->idle_ns, idle_ns);
    atomicAdd(&p.sstat->iters, acc.iters);
    atomicAdd(&p.sstat->checks, acc.checks);
    atomicAdd(&p.sstat->checks_hungry, acc.checks_hungry);
    atomicMax(&p.sstat->max_task_ns, max_task);
  }
}

// Blocks of the search kernel that can be resident on one SM for this query
// size (registers, shared memory and warp slots), from the occupancy API.
template <int W, bool EN>
__global__ void __launch_bounds__(W * 32) k_search(SearchParams p) {
  search_body<W, EN ? 1 : 0>(p);
}

// The tail-counting variant keeps the plain kernel's resident blocks (three
// of 8 warps, two of 16) under a register bound.
template <int W>
__global__ void __launch_bounds__(W * 32, W == 16 ? 2 : 768 / (W * 32)) k_search_tail(SearchParams p) {
  search_body<W, 2>(p);
}

namespace {

// mode: 0 plain, 1 match sets, 2 tail counting
template <int W>
cudaError_t search_occupancy(int* nb, size_t smem, int mode) {
  if (mode == 2) {
    cudaFuncSetAttribute(k_search_tail<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(nb, k_search_tail<W>, W * 32, smem);
  }
  if (mode == 1) {
    cudaFuncSetAttribute(k_search<W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(nb, k_search<W, true>, W * 32, smem);
  }
  cudaFuncSetAttribute(k_search<W, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(nb, k_search<W, false>, W * 32, smem);
}

template <int W>
void search_launch(const SearchParams& p, uint32_t blocks, size_t smem, cudaStream_t s, int mode) {
  if (mode == 2) {
    cudaFuncSetAttribute(k_search_tail<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_search_tail<W><<<blocks, W * 32, smem, s>>>(p);
  } else if (mode == 1) {
    cudaFuncSetAttribute(k_search<W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_search<W, true><<<blocks, W * 32, smem, s>>>(p);
  } else {
    cudaFuncSetAttribute(k_search<W, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_search<W, false><<<blocks, W * 32, smem, s>>>(p);
  }
}

}  // namespace

// Blocks of the search kernel that can be resident on one SM for this query
// size (registers, shared memory and warp slots), from the occupancy API.
// `mode` selects the instantiation: 0 plain counting (and hashes), 1 match
// sets, 2 tail counting.
uint32_t search_max_blocks(uint32_t n_q, uint32_t warps, int mode) {
  const size_t smem = search_smem_bytes(n_q, warps);
  int nb = 0;
  cudaError_t e = cudaSuccess;
  switch (warps) {
    case 4: e = search_occupancy<4>(&nb, smem, mode); break;
    case 16: e = search_occupancy<16>(&nb, smem, mode); break;
    default: e = search_occupancy<8>(&nb, smem, mode); break;
  }
  if (e != cudaSuccess) { cudaGetLastError(); return 0; }
  return (uint32_t)nb;
}

int search_mode(const SearchParams& p) { return p.enum_buf ? 1 : (p.tail ? 2 : 0); }

void launch_search(const SearchParams& p, uint32_t n_q, uint32_t blocks, uint32_t warps, cudaStream_t s) {
  const size_t smem = search_smem_bytes(n_q, warps);
  if (p.q) k_search_prep<<<1, 1, 0, s>>>(p.q, p.n_tasks, p.task_cap, p.sstat, p.error);
  const int mode = search_mode(p);
  switch (warps) {
    case 4: search_launch<4>(p, blocks, smem, s, mode); break;
    case 16: search_launch<16>(p, blocks, smem, s, mode); break;
    default: search_launch<8>(p, blocks, smem, s, mode); break;
  }
}

__global__ void k_finalize(uint32_t B, const UpdInfo* info, const unsigned long long* count,
                           const unsigned long long* hash, const unsigned long long* bytes, const uint32_t* safe,
                           const unsigned int* stop, uint64_t cap, int want_hash, csm_result* out,
                           uint32_t mut_bytes, const unsigned long long* stamp) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  const UpdInfo u = info[s];
  csm_result r;
  r.pos = 0; r.neg = 0; r.hash = 0; r.work_bytes = 0; r.latency_ns = 0;
  r.status = CSM_ST_OK; r.safe = safe ? safe[s] : 1u;
  if ((u.flags & UF_INVALID) || !(u.flags & UF_VALID)) {
    r.status = (u.flags & UF_INVALID) ? CSM_ST_INVALID : CSM_ST_OK;  // vertex updates count nothing
    r.safe = 1;
  } else {
    unsigned long long c = count[s];
    if (cap && c >= cap) { c = cap; r.status = CSM_ST_CAPPED; }
    else if (stop && stop[s] == kStopDeadline) r.status = CSM_ST_TIMED_OUT;  // c is a lower bound
    if (u.flags & UF_ADD) r.pos = c; else r.neg = c;
    if (want_hash && r.status == CSM_ST_OK) r.hash = hash[s];
    r.work_bytes = (bytes ? bytes[s] : 0ull) + ((u.flags & UF_MUT) ? (unsigned long long)mut_bytes : 0ull);
  }
  if (stamp) r.latency_ns = global_ns() - stamp[0];
  out[s] = r;
}

__global__ void k_classify(uint64_t n, const csm_update* ups, DevGraph g, const Plan* plan, uint8_t* safe) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const csm_update u = ups[i];
  uint8_t sf = 1;
  if (u.id1 < g.n && u.id2 < g.n) {
    const uint32_t L1 = g.vlabel[u.id1], L2 = g.vlabel[u.id2];
    for (uint32_t a = 0; a < plan->n_anchor && sf; a++) {
      const PlanAnchor* A = &plan->anchors[a];
      const uint32_t el = fold_elabel(g, u.label);
      if (A->el == el && ((A->la == L1 && A->lb == L2) || (A->la == L2 && A->lb == L1))) sf = 0;
    }
  }
  safe[i] = sf;
}

}  // namespace csm
