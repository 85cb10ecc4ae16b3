// Seeded synthetic workloads: RMAT data graphs with i.i.d. labels, queries
// sampled by random walk from the data graph, and edge-update streams built
// from held-out edges plus deletions of existing edges.
//
// The reference measures on public datasets (Amazon, LiveJournal, Orkut; see
// docs/csm_dataset/download_dataset.md in the reference); none is available
// offline, so these generators stand in for them with the shapes named per
// workload (vertex count, average degree, label counts and distributions,
// query size and density, stream length and insert/delete mix).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "graph_io.h"

namespace csm {

struct QuerySpec {
  uint32_t size = 6;
  bool dense = true;               // all induced edges; else spanning tree + extra
  uint32_t extra_edges = 0;        // sparse only: induced non-tree edges added
  double min_avg_degree = 0.0;     // dense only: resample until 2|E|/|V| >= this
};

struct WorkloadSpec {
  std::string name = "custom";
  uint64_t seed = 1;
  uint32_t log2_n = 14;            // 2^log2_n vertices
  double avg_degree = 8.0;         // total unique undirected edges = n * avg_degree / 2
  double rmat_a = 0.57, rmat_b = 0.19, rmat_c = 0.19;  // d = 1 - a - b - c
  uint32_t n_vlabels = 4;
  double vlabel_zipf = 0.0;        // 0 = uniform, else Zipf(s)
  uint32_t n_elabels = 1;
  std::vector<QuerySpec> queries{QuerySpec{}};
  // stream
  uint64_t n_updates = 2000;
  double insert_fraction = 1.0;
  double holdout_fraction = 0.0;   // if > 0: held-out = fraction * E (else = #inserts)
  // > 0: also keep the data graph as it stands after the first snapshot_at
  // updates of the stream (Workload::snapshot), so that a run can start there
  uint64_t snapshot_at = 0;
};

struct Query {
  uint32_t n = 0;
  std::vector<uint32_t> vlabels;
  std::vector<uint32_t> edges;     // (a, b, label)
  std::vector<uint32_t> sample;    // data vertex each query vertex was sampled from
};

struct Workload {
  WorkloadSpec spec;
  EdgeList initial;                // data graph at the start of the stream
  std::vector<Update> stream;
  std::vector<Query> queries;
  uint64_t total_edges = 0;        // unique edges generated before the hold-out
  EdgeList snapshot;               // graph after stream[0 .. spec.snapshot_at) (when snapshot_at > 0)
};

// Presets for the named workloads ("c1".."c5"); returns false for an unknown name.
bool preset(const std::string& name, WorkloadSpec& spec);

// Builds the whole workload; deterministic for a given spec (any thread count).
bool generate(const WorkloadSpec& spec, Workload& w, std::string& err);

bool save_query_text(const std::string& path, const Query& q);

}  // namespace csm
