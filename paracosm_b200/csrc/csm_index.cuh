// Candidate index of the TurboFlux (DCG) and SymBi (DCS) plugins as flat
// device arrays: per query vertex u, a bitset d2[u] over data vertices
// (ParaCOSM/CSM/matching/SymBi/symbi.h:55-62: the d1 / d2 flags), kept as a
// sound filter for the whole batch (it holds on the batch's union graph).
#pragma once
#include <vector>

#include "csm_host.cuh"
#include "csm_kernels.cuh"

namespace csm {

struct IndexQuery {
  uint32_t n;
  const std::vector<uint32_t>* vlabels;
  const std::vector<std::vector<uint32_t>>* nbr;
  const std::vector<std::vector<uint32_t>>* elabel;
};

struct IndexState {
  int algo = CSM_ALGO_GRAPHFLOW;
  uint64_t* d2 = nullptr;     // [n_q][words] candidate bitsets (null: no index)
  uint64_t words = 0;
  uint64_t entries = 0, vertices = 0;
};

int index_build(IndexState& ix, DevMem& mem, const DevGraph& g, const IndexQuery& q, int algo, cudaStream_t st,
                uint64_t* launches);
int index_apply_insertions(IndexState& ix, const DevGraph& g, const uint64_t* ins_key, const unsigned int* n_ranges,
                           const VRange* ranges, cudaStream_t st, uint64_t* launches);
int index_apply_deletions(IndexState& ix, const DevGraph& g, const uint64_t* del_key, const unsigned int* n_ranges,
                          const VRange* ranges, cudaStream_t st, uint64_t* launches);
int index_vertex_update(IndexState& ix, const DevGraph& g, const csm_update* ups, cudaStream_t st, uint64_t* launches);
void index_stats(const IndexState& ix, uint64_t* entries, uint64_t* vertices);
void index_free(IndexState& ix, DevMem& mem);

}  // namespace csm
