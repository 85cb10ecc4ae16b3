// The reference's plugin surface over the CUDA engine.
//
// `matching` mirrors the virtual interface every ParaCOSM plugin implements
// (ParaCOSM/CSM/matching/matching.h:9-66) and the constructor arguments the
// csm driver passes (ParaCOSM/CSM/matching/main.cpp:740-757).  Each plugin
// name the driver accepts with -a maps to one engine algorithm:
//   parallel_graphflow, graphflow  -> CSM_ALGO_GRAPHFLOW (no index)
//   parallel_turboflux, turboflux  -> CSM_ALGO_TURBOFLUX (DCG over a spanning tree)
//   parallel_symbi, symbi          -> CSM_ALGO_SYMBI     (DCS over a DAG of all query edges)
//   parallel_calig, calig          -> CSM_ALGO_CALIG     (CaLiG-style lighting filter; the reference
//                                     ships CaLiG as its own program, matching/Parallel_CaLiG)
//   parallel_newsp, newsp          -> CSM_ALGO_NEWSP     (NewSP-style neighbour-label-frequency filter;
//                                     the reference's own driver is matching/Parallel_NewSP)
// Differences from the reference, all deliberate:
//   - errors never exit the process: the calls record a CSM_E* code, and
//     error() / error_text() report the first one;
//   - the plugin does not hold references to caller Graphs; it copies the
//     query and the initial data graph into the engine once (Preprocessing);
//   - besides the per-update calls (one launch sequence per update, the
//     "plain" form), ProcessUpdates() hands a whole run of updates to the
//     engine, which batches them with the sequential semantics of
//     SingleThreadUpdate (ParaCOSM/CSM/matching/main.cpp:628-674).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "csm_gpu.h"
#include "graph_io.h"

namespace csm {

struct GpuOptions {
  int device = 0;
  int mode = CSM_MODE_BATCHED;   // CSM_MODE_PLAIN: one update per launch sequence
  uint32_t max_batch = 65536;
  bool want_hash = false;
  bool turboflux_compat = false;
  uint32_t warps_per_block = 0, blocks_per_sm = 0;  // 0: engine defaults / autotuner
  uint32_t vertex_headroom = 0;
  uint64_t hbm_budget_bytes = 0;
  uint64_t deadline_ns = 0;
  uint32_t enum_capacity = 0;  // > 0: keep embeddings for PrintMatches (the reference's --print-enum)
  bool graphs = false;         // replay each batch size's launch sequence as a CUDA graph
  // further queries on the same data graph (NewSP's multi-query build reads a
  // directory of queries, ParaCOSM/CSM/matching/Parallel_NewSP/graph/graph.cpp:550-574);
  // each is attached as a standing query with this plugin's settings and the
  // per-update counts are summed over all queries
  std::vector<EdgeList> more_queries;
};

class matching {
 public:
  matching(const EdgeList& query, const EdgeList& data, size_t max_num_results, bool print_prep, bool print_enum,
           bool homo, int algorithm, const GpuOptions& opt);
  virtual ~matching();
  matching(const matching&) = delete;
  matching& operator=(const matching&) = delete;

  virtual void Preprocessing();
  virtual void InitialMatching();
  virtual void AddEdge(uint32_t v1, uint32_t v2, uint32_t label);
  virtual void RemoveEdge(uint32_t v1, uint32_t v2);
  virtual void AddVertex(uint32_t id, uint32_t label);
  virtual void RemoveVertex(uint32_t id);
  // true when no query edge matches the label triple (the update is "safe")
  virtual bool Classify(uint32_t v1, uint32_t v2, uint32_t label);

  void GetMemoryCost(size_t& num_edges, size_t& num_vertices);
  void GetNumInitialResults(size_t& n) const { n = num_initial_results_; }
  void GetNumPositiveResults(size_t& n) const { n = num_positive_results_; }
  void GetNumNegativeResults(size_t& n) const { n = num_negative_results_; }
  void PrintCounter() const {}

  // Runs `ups` in order as batches; out[i] is the result of ups[i].
  int ProcessUpdates(const std::vector<Update>& ups, std::vector<csm_result>& out);
  // Prints the embeddings of the last ProcessUpdates of n updates, update by
  // update, one "m0 m1 ... " line each (needs GpuOptions::enum_capacity).
  int PrintMatches(size_t n);

  int error() const { return err_; }
  const std::string& error_text() const { return err_text_; }
  csm_ctx* context() const { return ctx_; }
  int algorithm() const { return algo_; }

 protected:
  int check(int rc);
  void run_one(const Update& u);
  int add_attached(uint64_t first, size_t n, csm_result* out);

  const EdgeList& query_;
  const EdgeList& data_;
  size_t max_num_results_;
  bool print_preprocessing_results_, print_enumeration_results_, homomorphism_;
  int algo_;
  GpuOptions opt_;
  csm_ctx* ctx_ = nullptr;
  std::vector<csm_ctx*> attached_;  // contexts of opt_.more_queries
  size_t num_initial_results_ = 0, num_positive_results_ = 0, num_negative_results_ = 0;
  uint64_t seq_ = 0;  // sequence number of the next submitted update
  int err_ = CSM_OK;
  std::string err_text_;
};

class Parallel_Graphflow : public matching {
 public:
  Parallel_Graphflow(const EdgeList& q, const EdgeList& d, size_t max_results, bool print_prep, bool print_enum,
                     bool homo, const GpuOptions& opt)
      : matching(q, d, max_results, print_prep, print_enum, homo, CSM_ALGO_GRAPHFLOW, opt) {}
};

class Parallel_TurboFlux : public matching {
 public:
  Parallel_TurboFlux(const EdgeList& q, const EdgeList& d, size_t max_results, bool print_prep, bool print_enum,
                     bool homo, const GpuOptions& opt)
      : matching(q, d, max_results, print_prep, print_enum, homo, CSM_ALGO_TURBOFLUX, opt) {}
};

// The reference spells this class Parrllel_SymBi (ParaCOSM/CSM/matching/Parallel_SymBi/parallel.h).
class Parrllel_SymBi : public matching {
 public:
  Parrllel_SymBi(const EdgeList& q, const EdgeList& d, size_t max_results, bool print_prep, bool print_enum,
                 bool homo, const GpuOptions& opt)
      : matching(q, d, max_results, print_prep, print_enum, homo, CSM_ALGO_SYMBI, opt) {}
};

// CaLiG (ParaCOSM/CSM/matching/Parallel_CaLiG/parallel_calig.cpp) is a
// standalone program in the reference; behind this interface it takes the
// same inputs as the other plugins.  An insertion of a present edge counts 0.
class Parallel_CaLiG : public matching {
 public:
  Parallel_CaLiG(const EdgeList& q, const EdgeList& d, size_t max_results, bool print_prep, bool print_enum,
                 bool homo, const GpuOptions& opt)
      : matching(q, d, max_results, print_prep, print_enum, homo, CSM_ALGO_CALIG, opt) {}
};

// NewSP's CSMPP (ParaCOSM/CSM/matching/Parallel_NewSP/matching/CSMPP.h:8-183),
// run by its own driver in the reference (Parallel_NewSP/matching/main.cpp),
// which takes the csm options and processes the stream with the sequential
// semantics; behind this interface it takes the same inputs as the others.
class CSMPP : public matching {
 public:
  CSMPP(const EdgeList& q, const EdgeList& d, size_t max_results, bool print_prep, bool print_enum, bool homo,
        const GpuOptions& opt)
      : matching(q, d, max_results, print_prep, print_enum, homo, CSM_ALGO_NEWSP, opt) {}
};

// Plugin for an -a name, or nullptr for an unknown name.
matching* make_plugin(const std::string& name, const EdgeList& q, const EdgeList& d, size_t max_results,
                      bool print_prep, bool print_enum, bool homo, const GpuOptions& opt);

}  // namespace csm
