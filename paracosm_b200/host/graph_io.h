// Graph, query and update-stream containers and their file formats.
//
// Text formats are the reference's (ParaCOSM/CSM/README.md:44-80, parsed by
// Graph::LoadFromFile / Graph::LoadUpdateStream,
// ParaCOSM/CSM/graph/graph.cpp:217-285):
//   graph / query:  "t ..." lines skipped, "v <id> <label>", and any other
//                   leading token is an edge "e <a> <b> <label>".
//   stream:         "v|-v <id> <label>", "e <a> <b> <label>", and any other
//                   token is an edge deletion "-e <a> <b> <label>".
// Binary formats (written by the workload generator, little endian):
//   graph  "CSMG" u32 ver, u32 n, u64 m, u32 n_vlabels, u32 n_elabels,
//          u32 vlabels[n], u32 edges[3*m] (a, b, label)
//   stream "CSMU" u32 ver, u64 n, then n records of 4 x u32:
//          (type | is_add << 8), id1, id2, label     (type is 'v' or 'e')
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace csm {

struct EdgeList {
  uint32_t n = 0;                  // number of vertex slots (ids are < n)
  uint32_t n_vlabels = 0, n_elabels = 0;
  std::vector<uint32_t> vlabels;   // NOT_EXIST (0xffffffff) for absent ids
  std::vector<uint32_t> edges;     // (a, b, label) triples, each undirected edge once
  uint64_t num_edges() const { return edges.size() / 3; }
};

// Same 16-byte layout as csm_update in include/csm_gpu.h.
struct Update {
  uint8_t type;    // 'v' or 'e'
  uint8_t is_add;  // 1 insert, 0 delete
  uint16_t pad;
  uint32_t id1, id2, label;
};
static_assert(sizeof(Update) == 16, "Update is 16 bytes");

constexpr uint32_t kNotExist = 0xffffffffu;

// Text loaders follow the reference's token rules; they return false and fill
// `err` instead of exiting.  Duplicate edges in a graph file keep the first
// label (Graph::AddEdge is a no-op on an existing edge,
// ParaCOSM/CSM/graph/graph.cpp:63-64).
bool load_graph_text(const std::string& path, EdgeList& g, std::string& err);
bool load_stream_text(const std::string& path, std::vector<Update>& s, std::string& err);
bool load_graph_binary(const std::string& path, EdgeList& g, std::string& err);
bool load_stream_binary(const std::string& path, std::vector<Update>& s, std::string& err);
// Picks the binary or text loader by the file's first four bytes.
bool load_graph_any(const std::string& path, EdgeList& g, std::string& err);
bool load_stream_any(const std::string& path, std::vector<Update>& s, std::string& err);

bool save_graph_text(const std::string& path, const EdgeList& g);
bool save_stream_text(const std::string& path, const std::vector<Update>& s);
bool save_graph_binary(const std::string& path, const EdgeList& g);
bool save_stream_binary(const std::string& path, const std::vector<Update>& s);

// Removes self loops and duplicate undirected edges (first occurrence wins)
// and recomputes label counts.
void canonicalize(EdgeList& g);

}  // namespace csm
