// Internal device-side layout shared by the engine's translation units.
//
// Data graph in HBM: a label-partitioned dynamic CSR.
//   - Row v lives at pool[row_off[v] .. row_off[v] + row_cap[v]); its first
//     deg(v) slots hold neighbour ids, grouped by "combo" = (neighbour vertex
//     label, edge label) and sorted by id inside each group, so the segment
//     S(v, a, l) (neighbours of v with vertex label a over edges labelled l)
//     is contiguous.  The remaining row_cap - deg slots are slack for
//     insertions; a row that outgrows its slack is moved to fresh pool space.
//   - dir[v * (NC + 1) + c] is the offset of combo c's segment inside row v
//     (dir[..NC] = deg(v)), so a segment is found with two 4-byte loads.
//   - Two pools alternate: when the active pool cannot absorb a batch's
//     relocations, every row is copied to the other pool with fresh slack.
// Edge updates of one batch are applied to the CSR before the search (the
// "union graph"), and each edge inserted or deleted inside the batch gets a
// temporal entry (its presence intervals in update-sequence numbers), so
// every update of the batch sees exactly the graph the sequential order
// gives it (ParaCOSM/CSM/matching/main.cpp:628-674).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/csm_gpu.h"

namespace csm {

constexpr uint32_t kNone = 0xffffffffu;
constexpr int32_t kTimeInf = 0x7fffffff;
constexpr uint32_t kMaxQ = 32;        // max query vertices
constexpr uint32_t kMaxQE = 256;      // max query edges
constexpr uint32_t kMaxBack = 32;     // backward entries per position
constexpr uint32_t kMaxBatch = 65536;

__host__ __device__ inline uint64_t mix64(uint64_t x) {  // MurmurHash3 fmix64
  x ^= x >> 33; x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33; return x;
}
// Per (query vertex, data vertex) term of the order-independent match hash.
__host__ __device__ inline uint64_t pair_hash(uint32_t q, uint32_t v) {
  return mix64((((uint64_t)(q + 1)) << 32) ^ (uint64_t)v ^ 0x9E3779B97F4A7C15ULL);
}

// Packed sort key of a directed entry (x, combo, y): x in the top bits, then
// the combo, then y, so that sorting groups rows and orders each row by
// (combo, id).  Widths are fixed per context; ids are < 2^yb - 1 so that the
// all-ones key is a sentinel that sorts after every real entry.
struct KeyBits {
  uint32_t yb;  // bits of a vertex id
  uint32_t cb;  // bits of a combo
  __host__ __device__ uint64_t pack(uint32_t x, uint32_t c, uint32_t y) const {
    return ((uint64_t)x << (cb + yb)) | ((uint64_t)c << yb) | (uint64_t)y;
  }
  __host__ __device__ uint32_t x_of(uint64_t k) const { return (uint32_t)(k >> (cb + yb)); }
  __host__ __device__ uint32_t c_of(uint64_t k) const { return (uint32_t)((k >> yb) & ((1ULL << cb) - 1)); }
  __host__ __device__ uint32_t y_of(uint64_t k) const { return (uint32_t)(k & ((1ULL << yb) - 1)); }
  __host__ __device__ uint32_t total() const { return 2 * yb + cb; }
  __host__ __device__ uint64_t sentinel() const { return total() >= 64 ? ~0ULL : ((1ULL << total()) - 1); }
  // Real entries are below the sentinel; unused list slots hold the
  // sentinel or all ones (memset 0xff), both of which fail this test.
  __host__ __device__ bool real(uint64_t k) const { return k < sentinel(); }
};

// Bump allocators and flags of the two alternating row pools.
struct PoolState {
  unsigned long long top[2];  // next free slot of each pool
  unsigned long long need;    // relocation demand of the current batch
  uint32_t active;            // index of the active pool
  uint32_t compact;           // set when this batch must compact first
  uint32_t error;             // nonzero: internal error code (see kErr*)
  uint32_t pad;
};
enum : uint32_t { kErrNone = 0, kErrPoolFull = 1, kErrListOverflow = 2, kErrTaskOverflow = 3, kErrWaitTimeout = 4,
                  kErrBadTask = 5, kErrRingState = 6, kErrTaskGuard = 7, kErrRowState = 8, kErrEdgeTable = 9 };

// Device view of the dynamic CSR (pointers into device memory).
struct DevGraph {
  uint32_t* vlabel;      // [n_cap]
  uint64_t* row_off;     // [n_cap]  offset into the active pool
  uint32_t* row_cap;     // [n_cap]
  uint32_t* dir;         // [n_cap * (nc + 1)]
  uint32_t* pools[2];    // the two row pools
  PoolState* ps;
  // temporal entries of the current batch, sorted by packed key (x, combo, nbr)
  uint32_t* t_start;     // [n_cap]
  uint32_t* t_count;     // [n_cap]  0 = vertex untouched in this batch
  uint64_t* t_key;       // packed keys
  int2* t_span;          // presence interval [start, end] in batch sequence numbers
  uint64_t pool_cap;     // entries per pool
  // label folding: sorted distinct query labels; label i of the list maps
  // to i, every other label to the inert label (n_qv / n_qe)
  const uint32_t* qlab_v;
  const uint32_t* qlab_e;
  uint32_t n_qv, n_qe;
  uint32_t n, n_cap, n_vl, n_el, nc;  // n_vl = n_qv + 1, n_el = n_qe + 1
  KeyBits kb;
  // Edge table: every (edge, label) of the graph -- the union graph during a
  // batch -- as one key in an open-addressing hash set (linear probing), so
  // that "is x a neighbour of v over label l" is one probe instead of a
  // binary search in v's segment.  emask = slots - 1; 0: no table (ids of
  // 30 bits or more, or more than 16 folded edge labels).
  uint64_t* ekeys;
  uint64_t emask;
};

// Edge-table keys: the smaller endpoint (30 bits), the larger (30 bits), the
// folded edge label (4 bits); two values no key takes mark empty and deleted
// slots.
constexpr uint64_t kEdgeEmpty = ~0ULL, kEdgeTomb = ~0ULL - 1;
__host__ __device__ __forceinline__ uint64_t edge_key(uint32_t a, uint32_t b, uint32_t l) {
  const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
  return ((uint64_t)lo << 34) | ((uint64_t)hi << 4) | (uint64_t)l;
}
__device__ __forceinline__ uint64_t edge_slot(uint64_t key, uint64_t mask) {
  uint64_t x = key ^ (key >> 33);  // MurmurHash3 fmix64, as mix64
  x *= 0xff51afd7ed558ccdULL; x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
  return x & mask;
}
// Loads of data read once per use at random places (edge-table slots, filter
// words, driver segments): they may fill L1 but go first when L1 needs room,
// so they do not push out the lines that are reused -- the search's register
// spills and the plan.
__device__ __forceinline__ uint64_t ld_stream(const uint64_t* a) {
  uint64_t v;
  asm("ld.global.L1::evict_first.u64 %0, [%1];" : "=l"(v) : "l"(a));
  return v;
}
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* a) {
  uint32_t v;
  asm("ld.global.L1::evict_first.u32 %0, [%1];" : "=r"(v) : "l"(a));
  return v;
}

// Probe sequence from a slot already loaded (first = ekeys[slot]).
__device__ __forceinline__ bool edge_probe_rest(const DevGraph& g, uint64_t key, uint64_t slot, uint64_t first) {
  uint64_t k = first;
  for (uint64_t n = 0; n <= g.emask; n++) {
    if (k == key) return true;
    if (k == kEdgeEmpty) return false;
    slot = (slot + 1) & g.emask;
    k = ld_stream(g.ekeys + slot);
  }
  return false;
}

__device__ __forceinline__ uint32_t fold_label(const uint32_t* sorted, uint32_t n, uint32_t l) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (sorted[mid] < l) lo = mid + 1; else hi = mid;
  }
  return (lo < n && sorted[lo] == l) ? lo : n;
}
__device__ __forceinline__ uint32_t fold_vlabel(const DevGraph& g, uint32_t l) {
  return l == kNone ? kNone : fold_label(g.qlab_v, g.n_qv, l);
}
__device__ __forceinline__ uint32_t fold_elabel(const DevGraph& g, uint32_t l) { return fold_label(g.qlab_e, g.n_qe, l); }

__device__ __forceinline__ uint32_t combo_of(const DevGraph& g, uint32_t vl, uint32_t el) {
  return vl * g.n_el + el;
}

// Segment [lo, hi) of combo c in row v, as absolute pool offsets.
__device__ __forceinline__ void segment(const DevGraph& g, uint32_t v, uint32_t c, uint64_t& lo, uint64_t& hi) {
  const uint32_t* d = g.dir + (size_t)v * (g.nc + 1) + c;
  const uint64_t base = g.row_off[v];
  lo = base + d[0];
  hi = base + d[1];
}

// lower_bound over a sorted uint32 range; returns the first index with a[i] >= x.
__device__ __forceinline__ uint64_t lower_bound_u32(const uint32_t* a, uint64_t lo, uint64_t hi, uint32_t x) {
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool contains_u32(const uint32_t* a, uint64_t lo, uint64_t hi, uint32_t x) {
  uint64_t p = lower_bound_u32(a, lo, hi, x);
  return p < hi && a[p] == x;
}

// Finds edge (x, y) in the union graph; returns its folded label or kNone.
__device__ __forceinline__ uint32_t find_label(const DevGraph& g, const uint32_t* pool, uint32_t x, uint32_t y) {
  const uint32_t ly = g.vlabel[y];
  for (uint32_t l = 0; l < g.n_el; l++) {
    uint64_t lo, hi;
    segment(g, x, ly * g.n_el + l, lo, hi);
    if (contains_u32(pool, lo, hi, y)) return l;
  }
  return kNone;
}

// Is edge (v, w) with combo c present at batch time t?  Only called for
// edges found in the union graph; edges not touched in this batch are present.
__device__ __forceinline__ bool present_at(const DevGraph& g, uint32_t v, uint32_t c, uint32_t w, int32_t t) {
  const uint32_t cnt = g.t_count[v];
  if (cnt == 0) return true;
  const uint64_t key = g.kb.pack(v, c, w);
  uint32_t lo = g.t_start[v], hi = lo + cnt;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (g.t_key[mid] < key) lo = mid + 1; else hi = mid;
  }
  const uint32_t end = g.t_start[v] + cnt;
  if (lo >= end || g.t_key[lo] != key) return true;
  for (uint32_t i = lo; i < end && g.t_key[i] == key; i++) {
    int2 s = g.t_span[i];
    if (s.x <= t && t <= s.y) return true;
  }
  return false;
}

// Number of entries of segment (v, c) present at batch time t, given its
// union-graph bounds: entries touched in this batch and absent at t are
// subtracted (an entry may carry several presence intervals).
__device__ __forceinline__ uint32_t seg_size_at(const DevGraph& g, uint32_t v, uint32_t c, uint64_t lo, uint64_t hi,
                                                int32_t t) {
  uint32_t size = (uint32_t)(hi - lo);
  const uint32_t cnt = g.t_count[v];
  if (cnt == 0 || size == 0) return size;
  const uint32_t beg = g.t_start[v], end = beg + cnt;
  const uint64_t k0 = g.kb.pack(v, c, 0);
  uint32_t a = beg, b = end;
  while (a < b) {
    uint32_t mid = (a + b) >> 1;
    if (g.t_key[mid] < k0) a = mid + 1; else b = mid;
  }
  for (uint32_t i = a; i < end && g.kb.x_of(g.t_key[i]) == v && g.kb.c_of(g.t_key[i]) == c;) {
    const uint64_t key = g.t_key[i];
    bool present = false;
    for (; i < end && g.t_key[i] == key; i++) {
      const int2 sp = g.t_span[i];
      if (sp.x <= t && t <= sp.y) present = true;
    }
    if (!present) size--;
  }
  return size;
}

// ---- query plan ------------------------------------------------------
// One plan per anchor query edge: positions 0 and 1 are the anchor's end
// points, the others follow the GraphFlow order of that edge
// (ParaCOSM/CSM/matching/GraphFlow/graphflow.cpp:36-169).  Position d >= 2
// has back entries (earlier position, combo of the edge to it) and a mask of
// earlier positions with the same vertex label (injectivity).
struct PlanPos {
  uint8_t qv;          // query vertex at this position
  uint8_t nb;          // number of back entries
  uint16_t boff;       // first back entry in PlanAnchor::back_*
  uint32_t samelab;    // bitmask over earlier positions with the same label
};

// Independent tail of an order: positions tail_at + 1 .. n - 1 have no query
// edge among them and no vertex label more than kTailGroup times, so once
// positions 0 .. tail_at are matched the completions are a product over the
// tail's label groups of injective assignments, counted without enumerating
// them.  Groups are listed in order of their first position (gpos: the
// positions, group after group, ascending inside a group; gsize: sizes).
constexpr uint32_t kTailGroup = 3;

struct PlanAnchor {
  uint32_t la, lb, el;       // label triple of the anchor (pos 0 label, pos 1 label, edge label)
  uint32_t tree;             // the anchor is an edge of the TurboFlux spanning tree (compat deletions)
  uint32_t prefix_mask;      // positions 0 .. tail_at
  uint8_t tail_at;           // last position matched one by one before the tail; 0: no tail
  uint8_t n_groups;
  uint8_t pad_[2];
  uint8_t gsize[kMaxQ];
  uint8_t gpos[kMaxQ];
  PlanPos pos[kMaxQ];
  uint8_t back_pos[kMaxQE];
  uint16_t back_combo[kMaxQE];
};

struct Plan {
  uint32_t n;          // query vertices
  uint32_t n_anchor;   // query edges
  PlanAnchor anchors[kMaxQE];
};

// Root search task: one (update, anchor edge, orientation) seed.
struct Task {
  uint32_t upd;        // index of the update inside the batch (= its batch time)
  uint16_t anchor;
  uint8_t orient;      // 0: (v1, v2) -> positions (0, 1); 1: swapped
  uint8_t pad;
};

// Batch-level per-update working state.
struct UpdInfo {
  uint32_t v1, v2;     // endpoints as given
  uint32_t label;      // anchor label used for counting (existing label for deletions)
  uint32_t flags;      // bit0 valid edge update, bit1 insertion, bit2 mutation applied, bit3 invalid
};
// UF_DUP: an insertion of an edge that is present at that point of the batch
enum : uint32_t { UF_VALID = 1u, UF_ADD = 2u, UF_MUT = 4u, UF_INVALID = 8u, UF_DUP = 16u };

}  // namespace csm
