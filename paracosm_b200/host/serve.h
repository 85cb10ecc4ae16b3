// Serving loop: standing queries over one resident data graph, with edge
// updates arriving as a stream and admitted in continuous batches.
//
// The reference has no serving mode (one query per process, the whole stream
// read up front, ParaCOSM/CSM/matching/main.cpp:676-871).  This runtime keeps
// the graph, every query's plan and candidate index, and the search state in
// HBM for its whole life, and:
//   - admits updates as they arrive: whenever the device is free it takes
//     every update that has arrived and not been processed (up to the batch
//     limit) as the next batch, so the batch size follows the load;
//   - admits standing queries as they arrive (between batches), each with its
//     own plugin and cap, while the device memory they need fits the budget;
//     a query that does not fit is refused;
//   - runs every admitted query on each batch in one launch sequence of the
//     owning context: the mutations once, the queries' searches concurrently
//     on their own streams;
//   - records per-update latency from arrival to results on the host.
// Results do not depend on how arrivals fall into batches: the engine applies
// the sequential semantics inside a batch.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "csm_gpu.h"
#include "graph_io.h"

namespace csm {

struct ServeQuery {
  std::vector<uint32_t> vlabels, edges;  // query graph: labels, (a, b, label) triples
  int algorithm = CSM_ALGO_GRAPHFLOW;
  uint64_t max_results = 0;              // 0: no cap
  double arrive_s = 0;                   // when the query arrives (seconds after the start)
};

struct ServeConfig {
  int device = 0;
  uint32_t max_batch = 65536;
  uint64_t budget_bytes = 40ull << 30;   // device memory for queries and search state
  double rate = 1e5;                     // offered load: Poisson arrivals, updates per second
  uint64_t seed = 7;
  bool want_hash = false;
  bool graphs = true;                    // replay each batch size's launch sequence as a CUDA graph
  uint64_t deadline_ns = 0;              // per-update search time limit (0: none)
  double max_seconds = 0;                // stop admitting updates after this long (0: run the stream)
  // offered loads of a sweep: one segment of max_seconds per rate, one after
  // another on the same graph, queries and stream (empty: `rate` alone)
  std::vector<double> rates;
};

struct ServeQueryResult {
  bool admitted = false;
  uint64_t first = 0;                    // index of the first update this query saw
  std::vector<csm_result> results;       // one per update from `first` on
};

struct ServeStats {
  uint64_t updates = 0, batches = 0, max_batch_seen = 0;
  double elapsed_s = 0, sustained = 0;   // updates / elapsed
  double p50_us = 0, p99_us = 0, mean_batch = 0;
  uint64_t device_bytes = 0;             // owner + admitted queries
  uint32_t queries_admitted = 0, queries_refused = 0;
  uint64_t results = 0, incomplete = 0;  // (update, query) results, and those CAPPED or TIMED_OUT
};

// Runs the stream through the serving loop.  Returns CSM_OK or a CSM_E* code
// (text in csm_gpu_last_error() or `err`).  With cfg.rates, `sweep` receives
// one ServeStats per rate (each segment continues the stream where the last
// one stopped) and `stats` covers the whole run.
int serve(const EdgeList& data, const std::vector<Update>& stream, const std::vector<ServeQuery>& queries,
          const ServeConfig& cfg, std::vector<ServeQueryResult>& out, ServeStats& stats, std::string& err,
          std::vector<ServeStats>* sweep = nullptr);

}  // namespace csm
