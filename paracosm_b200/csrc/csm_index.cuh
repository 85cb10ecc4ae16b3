// Candidate index of the TurboFlux (DCG) and SymBi (DCS) plugins as flat
// device arrays.
//
// The reference keeps, per query vertex u, hash maps d1[u] / d2[u] over data
// vertices plus the counters n1 / np1 / n2 / nc2 that maintain them
// (ParaCOSM/CSM/matching/SymBi/symbi.h:55-75, symbi.cpp:259-469).  Their
// meaning, over a DAG of the query (SymBi: every query edge oriented by BFS
// from a root; TurboFlux: a spanning tree):
//   d1[u][v]: L(v) = L(u) and every DAG parent p of u has a neighbour w of v
//             over an edge labelled l(u, p) with d1[p][w];
//   d2[u][v]: d1[u][v] and every DAG child c has such a neighbour w with
//             d2[c][w].
// Here each flag family is a bitset [n_q][words] over data vertex ids, so a
// membership test in the search is one 8-byte load from an array that fits
// in L2.  Maintenance recomputes the flags only where they can change:
// endpoints of changed edges, and neighbours (through the label-partitioned
// CSR) of vertices whose flag changed at a DAG neighbour, level by level in
// DAG order.
//
// The CaLiG-style and NewSP-style plugins use the same machinery for their
// filters, in a "lighting" mode: the DAG has no parents and makes every
// query neighbour a child; d1 is the label test plus, per (vertex label, edge
// label) pair of u's query edges, at least as many neighbours of that pair as
// u has; d2 is d1 with every query neighbour supported by a d1 neighbour.
// Both levels are functions of the graph and monotone in its edges.  d2
// contains CaLiG's lighting (ParaCOSM/CSM/matching/Parallel_CaLiG/
// parallel_calig.cpp:337-429: distinct lit witnesses for every query
// neighbour) and is that plugin's filter.  d1 implies NewSP's index check
// (ParaCOSM/CSM/matching/Parallel_NewSP/matching/CSMPP.cpp:81-113: at
// least as many neighbours of each vertex label and of each edge label) and
// is that plugin's filter.
//
// Every batch first brings the flags to the batch's union graph
// (a superset of the graph any of its updates sees, and the flags are
// monotone in the edge set, so d2 stays a sound filter for all of them), and
// to the graph after the batch once its deletions are applied.
#pragma once
#include <vector>

#include "csm_host.cuh"
#include "csm_kernels.cuh"

namespace csm {

struct IndexQuery {
  uint32_t n;
  const std::vector<uint32_t>* vlabels;            // folded query vertex labels
  const std::vector<std::vector<uint32_t>>* nbr;   // sorted adjacency
  const std::vector<std::vector<uint32_t>>* elabel;  // folded edge labels, parallel to nbr
  bool homo = false;  // homomorphism: the lighting filter asks one neighbour per (label, edge label) pair
};

// Query DAG in device memory.
struct IxDag {
  uint32_t nq;
  uint32_t n_edges;                  // DAG edges (parent, child)
  uint32_t qlab[kMaxQ];              // folded vertex label of each query vertex
  uint32_t npar[kMaxQ], nchd[kMaxQ];
  uint8_t par[kMaxQ][kMaxQ], chd[kMaxQ][kMaxQ];
  uint16_t par_vcombo[kMaxQ][kMaxQ];  // combo (L(p), l(u,p)): from a vertex of u to its parent-side neighbours
  uint16_t par_ucombo[kMaxQ][kMaxQ];  // combo (L(u), l(u,p)): from a vertex of p to its u-side neighbours
  uint16_t chd_vcombo[kMaxQ][kMaxQ];  // combo (L(c), l(u,c))
  uint16_t chd_ucombo[kMaxQ][kMaxQ];  // combo (L(u), l(u,c))
  uint8_t ep[kMaxQE], ec[kMaxQE];    // DAG edge list: parent, child
  uint16_t eel[kMaxQE];              // folded edge label
  // lighting mode: d2 draws its support from the children's d1, and d1
  // requires req_mult[u][i] neighbours in combo req_combo[u][i]
  uint32_t lighting;
  uint32_t nreq[kMaxQ];
  uint16_t req_combo[kMaxQ][kMaxQ];
  uint8_t req_mult[kMaxQ][kMaxQ];
};

// Flag bitsets: [n_q][words] each.  m1 / m2 mark vertices to re-evaluate,
// c1 / c2 record flags that changed in the current maintenance round.
struct IxBits {
  uint64_t *d1, *d2, *m1, *m2, *c1, *c2;
  uint64_t words;
  unsigned int* active;  // nonzero when the current round marked anything; else its kernels return at once
};

// Query vertices in DAG order, by value for a kernel argument.
struct IxOrder {
  uint32_t nq;
  uint32_t order[kMaxQ];
};

struct IndexState {
  int algo = CSM_ALGO_GRAPHFLOW;
  uint32_t coop_blocks = 0;  // grid of the single-launch round (0: not sized yet)
  bool active = false;
  uint64_t* d2 = nullptr;     // == bits.d2 (null: no index)
  uint64_t words = 0;
  IxBits bits{};
  IxDag h_dag{};
  IxDag* d_dag = nullptr;
  uint64_t* d_pop = nullptr;  // popcount scratch
  uint32_t root = 0;
  std::vector<uint32_t> order;
  int sm_count = 148;
  uint64_t entries = 0, vertices = 0;
};

int index_build(IndexState& ix, DevMem& mem, const DevGraph& g, const IndexQuery& q, int algo, int sm_count,
                cudaStream_t st, uint64_t* launches);
// Brings the flags to the CSR as it is now, after the directed entries in
// keys[0, L) (packed (x, combo, y), sentinel-padded) changed.
int index_apply_edges(IndexState& ix, const DevGraph& g, const uint64_t* keys, uint32_t L, cudaStream_t st,
                      uint64_t* launches);
// The same for the two directed entries keys[0..1] of one edge update, in two
// launches: the marks, then every propagation and re-evaluation step in one
// cooperative kernel.
int index_apply_edge_one(IndexState& ix, const DevGraph& g, const uint64_t* keys, cudaStream_t st,
                         uint64_t* launches);
int index_vertex_update(IndexState& ix, const DevGraph& g, const csm_update& h, cudaStream_t st, uint64_t* launches);
int index_counts(IndexState& ix, cudaStream_t st, uint64_t* d1_count, uint64_t* d2_count);
void index_stats(const IndexState& ix, uint64_t* entries, uint64_t* vertices);
void index_free(IndexState& ix, DevMem& mem);

}  // namespace csm
