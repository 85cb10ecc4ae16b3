// Candidate index of the TurboFlux / SymBi plugins (see csm_index.cuh).
#include "csm_index.cuh"

namespace csm {

int index_build(IndexState& ix, DevMem& mem, const DevGraph& g, const IndexQuery& q, int algo, cudaStream_t st,
                uint64_t* launches) {
  (void)mem; (void)g; (void)q; (void)st; (void)launches;
  ix.algo = algo;
  ix.d2 = nullptr;
  ix.words = 0;
  return CSM_OK;
}

int index_apply_insertions(IndexState& ix, const DevGraph& g, const uint64_t* ins_key, const unsigned int* n_ranges,
                           const VRange* ranges, cudaStream_t st, uint64_t* launches) {
  (void)ix; (void)g; (void)ins_key; (void)n_ranges; (void)ranges; (void)st; (void)launches;
  return CSM_OK;
}

int index_apply_deletions(IndexState& ix, const DevGraph& g, const uint64_t* del_key, const unsigned int* n_ranges,
                          const VRange* ranges, cudaStream_t st, uint64_t* launches) {
  (void)ix; (void)g; (void)del_key; (void)n_ranges; (void)ranges; (void)st; (void)launches;
  return CSM_OK;
}

int index_vertex_update(IndexState& ix, const DevGraph& g, const csm_update* ups, cudaStream_t st, uint64_t* launches) {
  (void)ix; (void)g; (void)ups; (void)st; (void)launches;
  return CSM_OK;
}

void index_stats(const IndexState& ix, uint64_t* entries, uint64_t* vertices) {
  *entries = ix.entries;
  *vertices = ix.vertices;
}

void index_free(IndexState& ix, DevMem& mem) {
  (void)mem;
  ix.d2 = nullptr;
}

}  // namespace csm
