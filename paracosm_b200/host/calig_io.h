// CaLiG's own file formats and its insertion-skip rule.
//
// The reference ships CaLiG as a separate program
// (ParaCOSM/CSM/matching/Parallel_CaLiG/parallel_calig.cpp, formats in
// ParaCOSM/CSM/matching/CaLiG/README.md):
//   query / data graph:  "v <id> <label>" and "e <a> <b>" (no edge labels);
//   stream:              "e <a> <b>" inserts (a, b), "e <-a-1> <-b-1>" deletes it.
// Loaded here with edge label 0.  inputQ (:101-143) maps a query label of -1
// to 0.  inputG (:271-335) sizes the graph by the largest vertex id and drops
// edges whose endpoint has no vertex line; vertices whose label the query
// does not use cannot take part in a match, which the engine's label folding
// already gives.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "graph_io.h"

namespace csm {

bool load_calig_graph(const std::string& path, EdgeList& g, std::string& err);
bool load_calig_stream(const std::string& path, std::vector<Update>& s, std::string& err, uint64_t max_updates = 0);
bool save_calig_graph(const std::string& path, const EdgeList& g);
bool save_calig_stream(const std::string& path, const std::vector<Update>& s);

// The reference's insertion loop (updateAndMatching, :1214-1272) skips an
// insertion when turnOnProcess_safe (:774-802) finds no candidate-neighbour
// entry at its first endpoint.  Such entries exist at a vertex that had a
// neighbour with a query label in the initial graph, and appear at a vertex
// once it is the second endpoint of an insertion the loop processed.  A
// skipped edge is still added to the neighbour sets, so a later insertion of
// it is a duplicate, but it never enters the candidate sets the search reads,
// so no later update finds matches through it.
//
// skip[i] = 1 marks the updates that rule skips (insertions between vertices
// with query labels; other updates are left alone).  The rule is a function
// of the stream, the initial graph and the query's labels; it matches the
// reference wherever the reference's lighting state does not itself lose
// matches.
std::vector<uint8_t> calig_skipped_insertions(const EdgeList& query, const EdgeList& data,
                                              const std::vector<Update>& stream);

}  // namespace csm
