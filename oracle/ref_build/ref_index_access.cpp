// Reads the candidate index (root, DAG, d1 / d2 flags) out of the reference's
// sequential SymBi and TurboFlux plugin objects, so that the oracle's
// restatement of that index can be pinned to the reference's own state.
//
// Test infrastructure only.  The plugin classes keep these members private
// (ParaCOSM/CSM/matching/SymBi/symbi.h:33-78, TurboFlux/turboflux.h:13-70);
// this one translation unit re-opens the access specifiers while including
// the unmodified headers.  Access specifiers do not change the layout of
// these classes, so the objects compiled from the reference sources are read
// as they are.
#include <algorithm>
#include <cstdio>
#include <iostream>
#include <queue>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

// everything the two plugin headers include, with normal access
#include "graph/graph.h"
#include "graph/storage_hash_map.hpp"
#include "matching/matching.h"
#include "utils/globals.h"
#include "utils/types.h"

#define private public
#include "matching/SymBi/symbi.h"
#include "matching/TurboFlux/turboflux.h"
#undef private

namespace {

template <class P>
void dump(P* p, uint32_t nq, FILE* f, long at) {
  fprintf(f, "at %ld\nroot %u\norder", at, p->q_root_);
  for (uint32_t i = 0; i < nq; i++) fprintf(f, " %u", p->serialized_tree_[i]);
  fprintf(f, "\n");
  for (uint32_t u = 0; u < nq; u++) {
    fprintf(f, "parents %u", u);
    std::vector<uint> b = p->treeNode_[u].backwards_;
    std::sort(b.begin(), b.end());
    for (uint x : b) fprintf(f, " %u", x);
    fprintf(f, "\n");
  }
  for (int which = 1; which <= 2; which++)
    for (uint32_t u = 0; u < nq; u++) {
      std::vector<uint> vs;
      for (const auto& kv : (which == 1 ? p->d1[u] : p->d2[u]))
        if (kv.second) vs.push_back(kv.first);
      std::sort(vs.begin(), vs.end());
      fprintf(f, "d%d %u", which, u);
      for (uint v : vs) fprintf(f, " %u", v);
      fprintf(f, "\n");
    }
}

}  // namespace

bool ref_dump_index(matching* m, const std::string& algo, uint32_t nq, FILE* f, long at) {
  if (algo == "symbi") { dump(static_cast<SymBi*>(m), nq, f, at); return true; }
  if (algo == "turboflux") { dump(static_cast<TurboFlux*>(m), nq, f, at); return true; }
  return false;
}
