// Data-graph kernels: load-time CSR build, per-batch resolution of edge
// lifetimes, in-place slack-block insertion / deletion, pool compaction.
//
// Reference semantics restated here:
//   Graph::AddEdge  (ParaCOSM/CSM/graph/graph.cpp:58-93)  sorted insert, duplicate = no-op
//   Graph::RemoveEdge (ParaCOSM/CSM/graph/graph.cpp:95-116) sorted erase, missing edge = error
//   Graph::GetEdgeLabel (ParaCOSM/CSM/graph/graph.cpp:133-174) label of an existing edge
#include "csm_kernels.cuh"

namespace csm {

// ---------------------------------------------------------------------
// load-time CSR build
// ---------------------------------------------------------------------

__global__ void k_load_edge_keys(const uint32_t* e, uint64_t m, const uint32_t* vlabel, uint32_t n,
                                 uint64_t* key, uint64_t* idx, unsigned long long* bad) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t a = e[3 * i], b = e[3 * i + 1];
  idx[i] = i;
  if (a == b) { key[i] = ~0ULL; return; }  // self loops are dropped
  if (a >= n || b >= n || vlabel[a] == kNone || vlabel[b] == kNone) {
    key[i] = ~0ULL;
    atomicAdd(bad, 1ULL);
    return;
  }
  key[i] = ((uint64_t)min(a, b) << 32) | (uint64_t)max(a, b);
}

// Folds raw vertex labels to the engine's compact labels (see DevGraph).
__global__ void k_fold_vlabels(uint32_t* vlabel, uint32_t n, DevGraph g) {
  uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  vlabel[v] = fold_vlabel(g, vlabel[v]);
}

// One directed entry pair per distinct undirected edge; repeats (same
// endpoints, later in the input) are dropped, so the first label wins.
__global__ void k_load_directed(const uint64_t* ukey, const uint64_t* uidx, uint64_t m, const uint32_t* e,
                                DevGraph g, uint64_t* dkey) {
  const KeyBits kb = g.kb;
  const uint32_t* vlabel = g.vlabel;
  const uint32_t n_el = g.n_el;
  uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint64_t k = ukey[j];
  if (k == ~0ULL || (j > 0 && ukey[j - 1] == k)) {
    dkey[2 * j] = kb.sentinel();
    dkey[2 * j + 1] = kb.sentinel();
    return;
  }
  const uint64_t i = uidx[j];
  const uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k, l = fold_elabel(g, e[3 * i + 2]);
  dkey[2 * j] = kb.pack(x, vlabel[y] * n_el + l, y);
  dkey[2 * j + 1] = kb.pack(y, vlabel[x] * n_el + l, x);
}

// Per (vertex, combo) run lengths (into dir, scanned later) and the first
// position of each vertex in the sorted keys.
__global__ void k_load_count(const uint64_t* dkey, uint64_t M, KeyBits kb, uint32_t nc, uint32_t* dir,
                             uint64_t* first, unsigned long long* n_valid) {
  uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  const uint64_t k = dkey[j];
  if (!kb.real(k)) return;
  const uint32_t x = kb.x_of(k), c = kb.c_of(k);
  if ((j + 1 == M) || !kb.real(dkey[j + 1])) *n_valid = j + 1;
  const bool head_x = (j == 0) || kb.x_of(dkey[j - 1]) != x;
  if (head_x) first[x] = j;
  const bool head_c = head_x || kb.c_of(dkey[j - 1]) != c;
  if (head_c) {
    uint64_t t = j;  // walk to the end of this (x, c) run
    while (t + 1 < M && kb.real(dkey[t + 1]) && kb.x_of(dkey[t + 1]) == x && kb.c_of(dkey[t + 1]) == c) t++;
    dir[(size_t)x * (nc + 1) + c] = (uint32_t)(t - j + 1);
  }
}

__device__ __forceinline__ uint32_t slack_cap(uint32_t d) { return d == 0 ? 0u : d + max(2u, d >> 2); }
__device__ __forceinline__ uint32_t grow_cap(uint32_t d) { return d + max(8u, d >> 1); }

__global__ void k_load_caps(const uint32_t* dir, uint32_t n_cap, uint32_t nc, uint32_t* cap, uint64_t* cap64) {
  uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n_cap) return;
  const uint32_t c = slack_cap(dir[(size_t)v * (nc + 1) + nc]);
  cap[v] = c;
  cap64[v] = c;
}

__global__ void k_load_scatter(const uint64_t* dkey, uint64_t M, KeyBits kb, const uint64_t* first,
                               const uint64_t* row_off, uint32_t* pool) {
  uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  const uint64_t k = dkey[j];
  if (!kb.real(k)) return;
  const uint32_t x = kb.x_of(k);
  pool[row_off[x] + (j - first[x])] = kb.y_of(k);
}

// Turns per-combo counts into row-relative segment offsets; dir[nc] = degree.
__global__ void k_dir_scan(uint32_t* dir, uint32_t n_cap, uint32_t nc) {
  uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n_cap) return;
  uint32_t* d = dir + (size_t)v * (nc + 1);
  uint32_t run = 0;
  for (uint32_t c = 0; c < nc; c++) { uint32_t t = d[c]; d[c] = run; run += t; }
  d[nc] = run;
}

// ---------------------------------------------------------------------
// batch preparation
// ---------------------------------------------------------------------

__global__ void k_batch_init(const csm_update* ups, uint32_t B, DevGraph g, uint64_t* ukey, uint32_t* useq,
                             UpdInfo* info) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  const csm_update u = ups[s];
  UpdInfo inf;
  inf.v1 = u.id1; inf.v2 = u.id2; inf.label = fold_elabel(g, u.label); inf.flags = 0;
  useq[s] = s;
  uint64_t key = ~0ULL;
  if (u.type == 'e') {
    const bool ok = u.id1 < g.n && u.id2 < g.n && u.id1 != u.id2 && g.vlabel[u.id1] != kNone &&
                    g.vlabel[u.id2] != kNone;
    if (ok) {
      key = ((uint64_t)min(u.id1, u.id2) << 32) | (uint64_t)max(u.id1, u.id2);
      inf.flags = UF_VALID | (u.is_add ? UF_ADD : 0u);
    } else {
      inf.flags = UF_INVALID;
    }
  }
  ukey[s] = key;
  info[s] = inf;
}

__device__ __forceinline__ void emit2(uint64_t* key, unsigned int* n, uint32_t cap, uint64_t k1, uint64_t k2,
                                      uint64_t* val, uint64_t v, unsigned int* err) {
  unsigned int i = atomicAdd(n, 2u);
  if (i + 2 > cap) { atomicExch(err, kErrListOverflow); return; }
  key[i] = k1; key[i + 1] = k2;
  if (val) { val[i] = v; val[i + 1] = v; }
}

// One thread per distinct edge key of the batch walks that edge's updates in
// sequence order, starting from its state before the batch.  It decides each
// update's effect (insert, duplicate insert, delete, delete of a missing
// edge), the label a deletion counts with, the presence intervals of the
// edge inside the batch, and the row insertions (before the search) and row
// deletions (after it) that turn the CSR into the union graph and back.
__global__ void k_resolve(const uint64_t* skey, const uint32_t* sseq, uint32_t B, DevGraph g,
                          const csm_update* ups, UpdInfo* info, ResolveOut out) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= B) return;
  const uint64_t k = skey[j];
  if (k == ~0ULL || (j > 0 && skey[j - 1] == k)) return;
  const uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k;
  const uint32_t lx = g.vlabel[x], ly = g.vlabel[y];
  const uint32_t* pool = g.pools[g.ps->active];
  const uint32_t l0 = find_label(g, pool, x, y);
  const bool present0 = (l0 != kNone);
  bool cur_p = present0;
  uint32_t cur_l = present0 ? l0 : 0u;
  int32_t cur_s = -1;
  uint64_t ins_mask = 0;
  unsigned int* err = &g.ps->error;
  for (uint32_t e = j; e < B && skey[e] == k; e++) {
    const uint32_t s = sseq[e];
    UpdInfo inf = info[s];
    const uint32_t label = inf.label;  // folded in k_batch_init
    if (inf.flags & UF_ADD) {
      if (cur_p) {
        inf.label = label;  // duplicate insert: graph unchanged, counted with the given label
        inf.flags |= UF_DUP;
      } else {
        cur_p = true; cur_l = label; cur_s = (int32_t)s;
        inf.label = label; inf.flags |= UF_MUT;
        if (!(present0 && label == l0)) ins_mask |= 1ULL << label;
      }
    } else {
      if (!cur_p) {
        inf.flags |= UF_INVALID;  // deleting a missing edge
      } else {
        inf.label = cur_l; inf.flags |= UF_MUT;
        const uint64_t span = (uint64_t)(uint32_t)cur_s | ((uint64_t)(uint32_t)s << 32);
        emit2(out.t_key, out.n_t, out.cap, g.kb.pack(x, ly * g.n_el + cur_l, y), g.kb.pack(y, lx * g.n_el + cur_l, x),
              out.t_span, span, err);
        cur_p = false;
      }
    }
    info[s] = inf;
  }
  if (cur_p && cur_s >= 0) {
    const uint64_t span = (uint64_t)(uint32_t)cur_s | ((uint64_t)(uint32_t)kTimeInf << 32);
    emit2(out.t_key, out.n_t, out.cap, g.kb.pack(x, ly * g.n_el + cur_l, y), g.kb.pack(y, lx * g.n_el + cur_l, x),
          out.t_span, span, err);
  }
  for (uint64_t m = ins_mask; m; m &= m - 1) {
    const uint32_t l = (uint32_t)__ffsll((long long)m) - 1;
    emit2(out.ins_key, out.n_ins, out.cap, g.kb.pack(x, ly * g.n_el + l, y), g.kb.pack(y, lx * g.n_el + l, x),
          nullptr, 0, err);
  }
  const uint64_t uni = ins_mask | (present0 ? (1ULL << l0) : 0ULL);
  const uint64_t endm = cur_p ? (1ULL << cur_l) : 0ULL;
  for (uint64_t m = uni & ~endm; m; m &= m - 1) {
    const uint32_t l = (uint32_t)__ffsll((long long)m) - 1;
    emit2(out.del_key, out.n_del, out.cap, g.kb.pack(x, ly * g.n_el + l, y), g.kb.pack(y, lx * g.n_el + l, x),
          nullptr, 0, err);
  }
}

// Appends one VRange per vertex run of a sorted packed-key list.  pad = 1
// marks a row longer than kBigRow entries before the batch: the mutation
// kernels give such rows a whole block instead of a warp.
__global__ void k_ranges(const uint64_t* key, uint32_t cap, KeyBits kb, VRange* ranges, unsigned int* n_ranges,
                         const uint32_t* dir, uint32_t nc) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cap) return;
  const uint64_t k = key[j];
  if (!kb.real(k)) return;
  const uint32_t x = kb.x_of(k);
  if (j > 0 && kb.x_of(key[j - 1]) == x) return;
  uint32_t t = j + 1;
  while (t < cap && kb.real(key[t]) && kb.x_of(key[t]) == x) t++;
  unsigned int i = atomicAdd(n_ranges, 1u);
  const uint32_t big = dir[(size_t)x * (nc + 1) + nc] > kBigRow ? 1u : 0u;
  ranges[i] = VRange{x, j, t - j, big};
}

__global__ void k_temporal_set(const VRange* ranges, const unsigned int* n_ranges, DevGraph g) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *n_ranges) return;
  const VRange r = ranges[i];
  g.t_start[r.x] = r.start;
  g.t_count[r.x] = r.count;
}

__global__ void k_temporal_clear(const VRange* ranges, const unsigned int* n_ranges, DevGraph g) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *n_ranges) return;
  g.t_count[ranges[i].x] = 0;
}

__global__ void k_reloc_need(const VRange* ranges, const unsigned int* n_ranges, DevGraph g) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long need = 0;
  if (i < *n_ranges) {
    const VRange r = ranges[i];
    const uint32_t deg = g.dir[(size_t)r.x * (g.nc + 1) + g.nc];
    if (deg + r.count > g.row_cap[r.x]) need = grow_cap(deg + r.count);
  }
  // warp-aggregated add
  for (int o = 16; o; o >>= 1) need += __shfl_down_sync(0xffffffffu, need, o);
  if ((threadIdx.x & 31) == 0 && need) atomicAdd(&g.ps->need, need);
}

__global__ void k_compact_check(DevGraph g) {
  PoolState* ps = g.ps;
  const unsigned long long free_slots = g.pool_cap - ps->top[ps->active];
  ps->compact = (ps->need > free_slots) ? 1u : 0u;
}

// Copies every row into the other pool with fresh slack (runs only when the
// active pool cannot absorb this batch's relocations).
__global__ void k_compact_copy(DevGraph g) {
  PoolState* ps = g.ps;
  if (!ps->compact) return;
  const uint32_t src = ps->active, dst = 1u - src;
  const uint32_t* sp = g.pools[src];
  uint32_t* dp = g.pools[dst];
  __shared__ unsigned long long base;
  __shared__ uint32_t scan[1024];
  for (uint64_t v0 = (uint64_t)blockIdx.x * blockDim.x; v0 < g.n_cap; v0 += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t v = v0 + threadIdx.x;
    uint32_t deg = 0, cap = 0;
    if (v < g.n_cap) { deg = g.dir[v * (g.nc + 1) + g.nc]; cap = slack_cap(deg); }
    scan[threadIdx.x] = cap;
    __syncthreads();
    for (uint32_t o = 1; o < blockDim.x; o <<= 1) {  // inclusive scan
      uint32_t t = threadIdx.x >= o ? scan[threadIdx.x - o] : 0;
      __syncthreads();
      scan[threadIdx.x] += t;
      __syncthreads();
    }
    if (threadIdx.x == blockDim.x - 1) base = atomicAdd(&ps->top[dst], (unsigned long long)scan[threadIdx.x]);
    __syncthreads();
    if (v < g.n_cap) {
      const uint64_t off = base + scan[threadIdx.x] - cap;
      if (off + cap > g.pool_cap) {
        atomicExch(&ps->error, kErrPoolFull);
      } else {
        const uint64_t so = g.row_off[v];
        for (uint32_t i = 0; i < deg; i++) dp[off + i] = sp[so + i];
        g.row_off[v] = off;
        g.row_cap[v] = cap;
      }
    }
    __syncthreads();
  }
}

__global__ void k_compact_finish(DevGraph g) {
  PoolState* ps = g.ps;
  if (ps->compact) {
    ps->top[ps->active] = 0;
    ps->active = 1u - ps->active;
    ps->compact = 0;
  }
  ps->need = 0;
}

// Combo of the row-relative entry index i: upper_bound(dir, i) - 1.
__device__ __forceinline__ uint32_t combo_at(const uint32_t* dirx, uint32_t nc, uint32_t i) {
  uint32_t lo = 0, hi = nc;  // find last c with dirx[c] <= i
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (dirx[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ uint32_t lower_bound_u64(const uint64_t* a, uint32_t lo, uint32_t hi, uint64_t x) {
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Group copies of n pool entries by G threads (a warp or a block).  Each
// round reads G entries into registers before any thread writes, so a move
// that overlaps its source is safe when left moves run front to back and
// right moves back to front.
template <int G>
__device__ __forceinline__ void group_sync() {
  if (G == 32) __syncwarp(); else __syncthreads();
}
template <int G>
__device__ __forceinline__ void group_move_left(uint32_t* pool, uint64_t src, uint64_t dst, uint32_t n,
                                                uint32_t lane) {
  for (uint32_t b = 0; b < n; b += G) {
    const uint32_t i = b + lane;
    uint32_t v = 0;
    if (i < n) v = pool[src + i];
    group_sync<G>();
    if (i < n) pool[dst + i] = v;
    group_sync<G>();
  }
}
template <int G>
__device__ __forceinline__ void group_move_right(uint32_t* pool, uint64_t src, uint64_t dst, uint32_t n,
                                                 uint32_t lane) {
  for (uint32_t b = n; b > 0;) {
    const uint32_t cnt = min((uint32_t)G, b);
    b -= cnt;
    uint32_t v = 0;
    if (lane < cnt) v = pool[src + b + lane];
    group_sync<G>();
    if (lane < cnt) pool[dst + b + lane] = v;
    group_sync<G>();
  }
}

// Merges each vertex's sorted insert list into its row; G = 32: one warp per
// row of at most kBigRow entries, G = blockDim: one block per longer row.
// Insert j (sorted by combo, then id) goes to row position p_j (its
// lower_bound in the old row); old entries in [p_j, p_{j+1}) then shift by
// j + 1, so the row moves as k + 1 contiguous blocks -- in place (last block
// first, back to front) or into a larger row elsewhere.
template <int G>
__global__ void k_mut_insert_g(const VRange* ranges, const unsigned int* n_ranges, const uint64_t* ins_key,
                               uint32_t* ins_dst, DevGraph g) {
  const uint32_t lane = threadIdx.x % G;
  const uint32_t groups_per_block = blockDim.x / G;
  const uint32_t nr = *n_ranges;
  PoolState* ps = g.ps;
  uint32_t* pool = g.pools[ps->active];
  __shared__ unsigned long long s_off[8];
  for (uint32_t w = blockIdx.x * groups_per_block + threadIdx.x / G; w - threadIdx.x / G < nr;
       w += gridDim.x * groups_per_block) {
    // every thread of a block-sized group walks the same w; warps of a
    // warp-sized group skip ranges of the other kind
    const bool mine = w < nr && ranges[w].pad == (G == 32 ? 0u : 1u);
    if (G == 32 && !mine) continue;
    if (G != 32 && !mine) { __syncthreads(); continue; }
    const VRange r = ranges[w];
    const uint32_t x = r.x, s = r.start, k = r.count;
    uint32_t* dirx = g.dir + (size_t)x * (g.nc + 1);
    const uint32_t deg = dirx[g.nc];
    const uint64_t off = g.row_off[x];
    const uint32_t new_deg = deg + k;
    uint64_t dst_off = off;
    uint32_t new_cap = 0;
    if (new_deg > g.row_cap[x]) {
      new_cap = grow_cap(new_deg);
      if (lane == 0) {
        unsigned long long o = atomicAdd(&ps->top[ps->active], (unsigned long long)new_cap);
        if (o + new_cap > g.pool_cap) { atomicExch(&ps->error, kErrPoolFull); o = ~0ULL; }
        s_off[threadIdx.x / G] = o;
      }
      group_sync<G>();
      dst_off = s_off[threadIdx.x / G];
      group_sync<G>();
      if (dst_off == ~0ULL) continue;  // uniform across the group
    }
    // 1. positions p_j in the old row
    for (uint32_t j = lane; j < k; j += G) {
      const uint64_t key = ins_key[s + j];
      const uint32_t c = g.kb.c_of(key), y = g.kb.y_of(key);
      ins_dst[s + j] = (uint32_t)lower_bound_u32(pool + off, dirx[c], dirx[c + 1], y);
    }
    group_sync<G>();
    // 2. old entries, block by block
    if (dst_off == off) {
      for (int64_t j = (int64_t)k - 1; j >= 0; j--) {
        const uint32_t a = ins_dst[s + j], b = (j + 1 < (int64_t)k) ? ins_dst[s + j + 1] : deg;
        if (b > a) group_move_right<G>(pool, off + a, off + a + (uint64_t)j + 1, b - a, lane);
      }
    } else {
      group_move_left<G>(pool, off, dst_off, ins_dst[s], lane);  // different rows: no overlap
      for (uint32_t j = 0; j < k; j++) {
        const uint32_t a = ins_dst[s + j], b = (j + 1 < k) ? ins_dst[s + j + 1] : deg;
        if (b > a) group_move_left<G>(pool, off + a, dst_off + a + j + 1, b - a, lane);
      }
    }
    // 3. inserted entries
    for (uint32_t j = lane; j < k; j += G) pool[dst_off + ins_dst[s + j] + j] = g.kb.y_of(ins_key[s + j]);
    group_sync<G>();
    // 4. directory: a combo's segment starts after the inserts of smaller combos
    for (uint32_t c = lane; c <= g.nc; c += G) {
      const uint32_t add = lower_bound_u64(ins_key, s, s + k, g.kb.pack(x, 0, 0) + ((uint64_t)c << g.kb.yb)) - s;
      dirx[c] += add;
    }
    if (lane == 0 && new_cap) { g.row_off[x] = dst_off; g.row_cap[x] = new_cap; }
    group_sync<G>();
  }
}

// Removes each vertex's sorted delete list from its row in place (G as
// above).  Delete j sits at row position q_j; the old entries between q_j and
// q_{j+1} move left by j + 1, blocks front to back.  `del_pos` is scratch of
// the delete list's length.
template <int G>
__global__ void k_mut_delete_g(const VRange* ranges, const unsigned int* n_ranges, const uint64_t* del_key,
                               uint32_t* del_pos, DevGraph g) {
  const uint32_t lane = threadIdx.x % G;
  const uint32_t groups_per_block = blockDim.x / G;
  const uint32_t nr = *n_ranges;
  uint32_t* pool = g.pools[g.ps->active];
  for (uint32_t w = blockIdx.x * groups_per_block + threadIdx.x / G; w - threadIdx.x / G < nr;
       w += gridDim.x * groups_per_block) {
    const bool mine = w < nr && ranges[w].pad == (G == 32 ? 0u : 1u);
    if (G == 32 && !mine) continue;
    if (G != 32 && !mine) { __syncthreads(); continue; }
    const VRange r = ranges[w];
    const uint32_t x = r.x, s = r.start, k = r.count;
    uint32_t* dirx = g.dir + (size_t)x * (g.nc + 1);
    const uint32_t deg = dirx[g.nc];
    const uint64_t off = g.row_off[x];
    for (uint32_t j = lane; j < k; j += G) {
      const uint64_t key = del_key[s + j];
      const uint32_t c = g.kb.c_of(key), y = g.kb.y_of(key);
      del_pos[s + j] = (uint32_t)lower_bound_u32(pool + off, dirx[c], dirx[c + 1], y);
    }
    group_sync<G>();
    for (uint32_t j = 0; j < k; j++) {
      const uint32_t a = del_pos[s + j] + 1, b = (j + 1 < k) ? del_pos[s + j + 1] : deg;
      if (a < j + 1 || a > deg) {  // a deleted entry missing from its row: leave the row, report
        if (lane == 0) atomicExch(&g.ps->error, kErrRowState);
        break;
      }
      if (b > a) group_move_left<G>(pool, off + a, off + a - (j + 1), b - a, lane);
    }
    for (uint32_t c = lane; c <= g.nc; c += G) {
      const uint32_t sub = lower_bound_u64(del_key, s, s + k, g.kb.pack(x, 0, 0) + ((uint64_t)c << g.kb.yb)) - s;
      dirx[c] -= sub;
    }
    group_sync<G>();
  }
}

// Both row kinds of a batch: rows up to kBigRow entries by warps, longer rows
// by 256-thread blocks.
void launch_mut_insert(const VRange* ranges, const unsigned int* n_ranges, const uint64_t* ins_key,
                       uint32_t* ins_dst, const DevGraph& g, uint32_t warp_blocks, uint32_t big_blocks,
                       cudaStream_t st) {
  k_mut_insert_g<32><<<warp_blocks, 256, 0, st>>>(ranges, n_ranges, ins_key, ins_dst, g);
  k_mut_insert_g<256><<<big_blocks, 256, 0, st>>>(ranges, n_ranges, ins_key, ins_dst, g);
}
void launch_mut_delete(const VRange* ranges, const unsigned int* n_ranges, const uint64_t* del_key,
                       uint32_t* del_pos, const DevGraph& g, uint32_t warp_blocks, uint32_t big_blocks,
                       cudaStream_t st) {
  k_mut_delete_g<32><<<warp_blocks, 256, 0, st>>>(ranges, n_ranges, del_key, del_pos, g);
  k_mut_delete_g<256><<<big_blocks, 256, 0, st>>>(ranges, n_ranges, del_key, del_pos, g);
}

// ------------------------------------------------------------ edge table

__device__ __forceinline__ void edge_insert(const DevGraph& g, uint64_t key) {
  uint64_t slot = edge_slot(key, g.emask);
  for (uint64_t n = 0; n <= g.emask; n++) {
    const uint64_t k = g.ekeys[slot];
    if (k == key) return;
    if (k == kEdgeEmpty) {
      const unsigned long long prev =
          atomicCAS((unsigned long long*)&g.ekeys[slot], (unsigned long long)kEdgeEmpty, (unsigned long long)key);
      if (prev == kEdgeEmpty || prev == key) return;  // placed here, or by another thread inserting the same key
    }
    slot = (slot + 1) & g.emask;
  }
  atomicExch(&g.ps->error, kErrEdgeTable);  // no empty slot left
}

__device__ __forceinline__ void edge_delete(const DevGraph& g, uint64_t key) {
  uint64_t slot = edge_slot(key, g.emask);
  for (uint64_t n = 0; n <= g.emask; n++) {
    const uint64_t k = g.ekeys[slot];
    if (k == key) {
      atomicCAS((unsigned long long*)&g.ekeys[slot], (unsigned long long)key, (unsigned long long)kEdgeTomb);
      return;
    }
    if (k == kEdgeEmpty) return;
    slot = (slot + 1) & g.emask;
  }
}

// One warp per row: the lanes take the row's entries 32 at a time and find
// each entry's combo by a binary search in the row's directory, so that a
// row's insertions run side by side (combos hold a few entries each: looping
// over combos left most lanes idle and the insertions one after another).
__global__ void k_edge_fill(DevGraph g) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t* pool = g.pools[g.ps->active];
  for (uint32_t v = warp; v < g.n; v += nwarps) {
    const uint32_t* dirv = g.dir + (size_t)v * (g.nc + 1);
    const uint32_t total = dirv[g.nc];
    if (total == 0) continue;
    const uint64_t off = g.row_off[v];
    for (uint32_t i = lane; i < total; i += 32) {
      uint32_t lo = 0, hi = g.nc - 1;  // the last combo c with dirv[c] <= i: its segment holds entry i
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (dirv[mid] <= i) lo = mid; else hi = mid - 1;
      }
      const uint32_t w = pool[off + i];
      if (v < w) edge_insert(g, edge_key(v, w, lo % g.n_el));
    }
  }
}

__global__ void k_edge_list(const uint64_t* keys, uint32_t L, DevGraph g, uint32_t del) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L) return;
  const uint64_t k = keys[i];
  if (!g.kb.real(k)) return;
  const uint32_t x = g.kb.x_of(k), y = g.kb.y_of(k);
  if (x >= y) return;
  const uint64_t ek = edge_key(x, y, g.kb.c_of(k) % g.n_el);
  if (del) edge_delete(g, ek); else edge_insert(g, ek);
}

// ------------------------------------------------- one update per launch
//
// The plain form runs each edge update on its own.  A batch of one needs no
// sorting, no grouping by edge and no temporal entries: an insertion is
// searched after its edge is added and a deletion before its edge is
// removed, so the graph at search time is the sequential one.  Its
// preparation is one kernel and its row mutation another (plus the
// compaction copy when an insertion's relocation does not fit).

__global__ void k_plain_resolve(const csm_update* up, DevGraph g, UpdInfo* info, uint64_t* keys, unsigned int* cnt,
                                unsigned long long* count, unsigned long long* hash, unsigned long long* bytes,
                                unsigned int* stop) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const csm_update u = *up;
  UpdInfo inf;
  inf.v1 = u.id1; inf.v2 = u.id2; inf.label = fold_elabel(g, u.label); inf.flags = 0;
  keys[0] = ~0ULL; keys[1] = ~0ULL;
  for (int i = 0; i < 16; i++) cnt[i] = 0;
  count[0] = 0; hash[0] = 0; bytes[0] = 0; stop[0] = 0;
  PoolState* ps = g.ps;
  ps->need = 0;
  ps->compact = 0;
  if (u.type == 'e') {
    const bool ok = u.id1 < g.n && u.id2 < g.n && u.id1 != u.id2 && g.vlabel[u.id1] != kNone &&
                    g.vlabel[u.id2] != kNone;
    if (!ok) {
      inf.flags = UF_INVALID;
    } else {
      inf.flags = UF_VALID | (u.is_add ? UF_ADD : 0u);
      const uint32_t l0 = find_label(g, g.pools[ps->active], u.id1, u.id2);
      const uint32_t x = min(u.id1, u.id2), y = max(u.id1, u.id2);
      if (u.is_add) {
        if (l0 != kNone) {
          inf.flags |= UF_DUP;  // graph unchanged; counted with the given label
        } else {
          inf.flags |= UF_MUT;
          keys[0] = g.kb.pack(x, g.vlabel[y] * g.n_el + inf.label, y);
          keys[1] = g.kb.pack(y, g.vlabel[x] * g.n_el + inf.label, x);
          unsigned long long need = 0;
          const uint32_t ends[2] = {x, y};
          for (int k = 0; k < 2; k++) {
            const uint32_t v = ends[k];
            const uint32_t deg = g.dir[(size_t)v * (g.nc + 1) + g.nc];
            if (deg + 1 > g.row_cap[v]) need += grow_cap(deg + 1);
          }
          ps->need = need;
          ps->compact = (need > g.pool_cap - ps->top[ps->active]) ? 1u : 0u;
        }
      } else if (l0 == kNone) {
        inf.flags |= UF_INVALID;  // deleting a missing edge
      } else {
        inf.label = l0;  // a deletion counts with the edge's own label
        inf.flags |= UF_MUT;
        keys[0] = g.kb.pack(x, g.vlabel[y] * g.n_el + l0, y);
        keys[1] = g.kb.pack(y, g.vlabel[x] * g.n_el + l0, x);
      }
    }
  }
  info[0] = inf;
}

__global__ void __launch_bounds__(256) k_plain_mutate(DevGraph g, const UpdInfo* info, const uint64_t* keys,
                                                      csm_result* out, const unsigned long long* stamp,
                                                      uint32_t mut_bytes) {
  PoolState* ps = g.ps;
  const uint32_t lane = threadIdx.x;
  __shared__ unsigned long long s_off;
  __shared__ uint32_t s_pos, s_bad;
  if (lane == 0) {
    if (ps->compact) {  // k_compact_copy moved every row to the other pool (k_compact_finish's step)
      ps->top[ps->active] = 0;
      ps->active = 1u - ps->active;
      ps->compact = 0;
    }
    ps->need = 0;
  }
  __syncthreads();
  const UpdInfo inf = info[0];
  uint32_t* pool = g.pools[ps->active];
  if (inf.flags & UF_MUT) {
    const bool add = (inf.flags & UF_ADD) != 0;
    for (int k = 0; k < 2; k++) {
      const uint64_t key = keys[k];
      const uint32_t x = g.kb.x_of(key), c = g.kb.c_of(key), y = g.kb.y_of(key);
      uint32_t* dirx = g.dir + (size_t)x * (g.nc + 1);
      const uint32_t deg = dirx[g.nc];
      const uint64_t off = g.row_off[x];
      if (lane == 0) {
        s_pos = (uint32_t)lower_bound_u32(pool + off, dirx[c], dirx[c + 1], y);
        s_bad = 0;
        if (!add && (s_pos >= dirx[c + 1] || pool[off + s_pos] != y)) s_bad = 1;  // the entry must be there
      }
      __syncthreads();
      const uint32_t p = s_pos;
      if (s_bad) {
        if (lane == 0) atomicExch(&ps->error, kErrRowState);
        break;
      }
      if (add) {
        uint64_t dst = off;
        uint32_t new_cap = 0;
        if (deg + 1 > g.row_cap[x]) {
          new_cap = grow_cap(deg + 1);
          if (lane == 0) {
            unsigned long long o = atomicAdd(&ps->top[ps->active], (unsigned long long)new_cap);
            if (o + new_cap > g.pool_cap) { atomicExch(&ps->error, kErrPoolFull); o = ~0ULL; }
            s_off = o;
          }
          __syncthreads();
          dst = s_off;
          if (dst == ~0ULL) break;  // the same value in every thread
          group_move_left<256>(pool, off, dst, p, lane);                 // different rows: no overlap
          group_move_left<256>(pool, off + p, dst + p + 1, deg - p, lane);
        } else {
          group_move_right<256>(pool, off + p, off + p + 1, deg - p, lane);
        }
        if (lane == 0) pool[dst + p] = y;
        for (uint32_t cc = c + 1 + lane; cc <= g.nc; cc += 256) dirx[cc] += 1;
        if (lane == 0 && new_cap) { g.row_off[x] = dst; g.row_cap[x] = new_cap; }
      } else {
        group_move_left<256>(pool, off + p + 1, off + p, deg - p - 1, lane);
        for (uint32_t cc = c + 1 + lane; cc <= g.nc; cc += 256) dirx[cc] -= 1;
      }
      __syncthreads();
    }
  }
  if (g.emask && (inf.flags & UF_MUT) && lane == 0) {  // the edge table follows the rows
    const uint64_t k0 = keys[0];
    const uint64_t ek = edge_key(g.kb.x_of(k0), g.kb.y_of(k0), g.kb.c_of(k0) % g.n_el);
    if (inf.flags & UF_ADD) edge_insert(g, ek); else edge_delete(g, ek);
  }
  if (out && lane == 0) {
    // an update whose label triple matches no query edge: nothing to count
    csm_result r;
    r.pos = 0; r.neg = 0; r.hash = 0;
    r.status = (inf.flags & UF_INVALID) ? CSM_ST_INVALID : CSM_ST_OK;
    r.safe = 1;
    r.work_bytes = (inf.flags & UF_MUT) ? (unsigned long long)mut_bytes : 0ull;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    r.latency_ns = stamp ? t - stamp[0] : 0ull;
    out[0] = r;
  }
}

// Vertex deletion: the packed keys of every directed entry incident to v,
// (v, combo, y) and (y, combo', v), for the deletion kernels.
__global__ void k_vdel_keys(DevGraph g, uint32_t v, uint32_t deg, uint64_t* keys) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= deg) return;
  const uint32_t* pool = g.pools[g.ps->active];
  const uint32_t* dirv = g.dir + (size_t)v * (g.nc + 1);
  const uint32_t y = pool[g.row_off[v] + i];
  const uint32_t c = combo_at(dirv, g.nc, i);
  const uint32_t el = c % g.n_el;
  keys[2 * i] = g.kb.pack(v, c, y);
  keys[2 * i + 1] = g.kb.pack(y, g.vlabel[v] * g.n_el + el, v);
}

// Vertex insertion (Graph::AddVertex, ParaCOSM/CSM/graph/graph.cpp:23-49): sets
// the label of an absent vertex slot.  A deletion of an id beyond the
// vertex slots is invalid; other deletions are applied by the caller.
__global__ void k_vertex_update(const csm_update* ups, uint32_t B, DevGraph g, UpdInfo* info) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  const csm_update u = ups[s];
  if (u.type != 'v') return;
  UpdInfo inf;
  inf.v1 = u.id1; inf.v2 = 0; inf.label = u.label; inf.flags = 0;
  if (u.is_add && u.id1 < g.n_cap) {
    if (g.vlabel[u.id1] == kNone) g.vlabel[u.id1] = fold_vlabel(g, u.label);
  } else if (u.is_add || u.id1 >= g.n) {
    inf.flags = UF_INVALID;
  }
  info[s] = inf;
}

}  // namespace csm
