/*
 * csm_gpu_plugin.h - the engine as a plugin of the reference's own driver.
 *
 * GpuPlugin derives from the reference's plugin base class `matching`
 * (ParaCOSM/CSM/matching/matching.h:9-66) and forwards every virtual method
 * to the C ABI in csm_gpu.h, so the reference's driver loop -- the sequential
 * SingleThreadUpdate (ParaCOSM/CSM/matching/main.cpp:628-674) or any other
 * caller of `matching*` -- runs the GPU engine unchanged.  It is compiled in
 * the reference's source tree: include it after the reference's headers are
 * on the include path (-I ParaCOSM/CSM) together with this directory, and
 * link -lcsmgpu.  A maintainer adds, beside the -a branches of
 * ParaCOSM/CSM/matching/main.cpp:740-757,
 *
 *   else if (algorithm == "gpu_symbi")
 *     mm = new GpuPlugin(query_graph, data_graph, max_num_results, print_prep, print_enum, homo,
 *                        CSM_ALGO_SYMBI);
 *
 * (and gpu_turboflux, gpu_graphflow, gpu_calig, gpu_newsp likewise).
 *
 * Conventions of the reference that the plugin keeps:
 *   - it holds references to the caller's query and data Graphs and keeps the
 *     data Graph current (Graph::AddEdge before an insertion is counted,
 *     Graph::RemoveEdge after a deletion is counted), as the reference's
 *     plugins do (e.g. ParaCOSM/CSM/matching/SymBi/symbi.cpp:679-965);
 *   - counts accumulate in the base class counters, read with
 *     GetNum{Initial,Positive,Negative}Results;
 *   - with print_enum, every embedding of an update is written to std::cout
 *     as one line of data vertices in query-vertex order, as the reference's
 *     sequential plugins do (ParaCOSM/CSM/matching/SymBi/symbi.cpp:564-569);
 *   - an engine error is printed and ends the process with exit(-1), the
 *     reference's error convention (ParaCOSM/CSM/graph/graph.cpp:98-109).
 * Each AddEdge / RemoveEdge / AddVertex / RemoveVertex is one submit of one
 * update (CSM_MODE_PLAIN, the plain form).  ProcessUpdates hands a run of
 * updates to the engine in one submit (CSM_MODE_BATCHED), with identical
 * counts.
 */
#ifndef CSM_GPU_PLUGIN_H
#define CSM_GPU_PLUGIN_H

#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "csm_gpu.h"
#include "graph/graph.h"
#include "matching/matching.h"

class GpuPlugin : public matching {
 public:
  // algorithm: CSM_ALGO_*; mode: CSM_MODE_PLAIN (one update per call) or
  // CSM_MODE_BATCHED (for ProcessUpdates); device: CUDA ordinal.
  GpuPlugin(Graph& query_graph, Graph& data_graph, size_t max_num_results, bool print_preprocessing_results,
            bool print_enumeration_results, bool homomorphism, int algorithm, int mode = CSM_MODE_PLAIN,
            int device = 0)
      : matching(query_graph, data_graph, max_num_results, print_preprocessing_results, print_enumeration_results,
                 homomorphism) {
    csm_cfg c;
    csm_gpu_default_cfg(&c);
    c.algorithm = algorithm;
    c.homomorphism = homomorphism ? 1 : 0;
    // the reference's plugins take `uint max_num_results` (main.cpp:682); UINT_MAX and above mean no cap
    c.max_results = max_num_results >= (size_t)UINT_MAX ? 0 : (uint64_t)max_num_results;
    c.mode = mode;
    c.device = device;
    c.want_hash = 0;
    // embeddings kept per submit for print_enum (the reference prints every one it finds)
    c.enum_capacity = print_enumeration_results ? kEnumCapacity : 0;
    check(csm_gpu_create(&c, &ctx_));
  }
  ~GpuPlugin() override { csm_gpu_destroy(ctx_); }

  // Copies the query and the current data graph into the engine and builds
  // the plugin's candidate index (the reference's Preprocessing builds its
  // DAG and index the same way, e.g. SymBi/symbi.cpp:113-402).
  void Preprocessing() override {
    std::vector<uint32_t> qv, qe, dv, de;
    flatten(query_, qv, qe);
    flatten(data_, dv, de);
    check(csm_gpu_set_query(ctx_, (uint32_t)qv.size(), qv.data(), (uint32_t)(qe.size() / 3), qe.data()));
    check(csm_gpu_load_graph(ctx_, (uint32_t)dv.size(), dv.data(), de.size() / 3, de.data()));
    check(csm_gpu_build_index(ctx_));
  }

  void InitialMatching() override {
    uint64_t c = 0;
    check(csm_gpu_initial_match(ctx_, &c));
    num_initial_results_ += c;
  }

  void AddEdge(uint v1, uint v2, uint label) override {
    data_.AddEdge(v1, v2, label);
    run_one('e', 1, v1, v2, label);
  }
  void RemoveEdge(uint v1, uint v2) override {
    run_one('e', 0, v1, v2, 0);
    data_.RemoveEdge(v1, v2);
  }
  void AddVertex(uint id, uint label) override {
    data_.AddVertex(id, label);
    run_one('v', 1, id, 0, label);
  }
  void RemoveVertex(uint id) override {
    run_one('v', 0, id, 0, 0);
    data_.RemoveVertex(id);
  }

  // true: no query edge matches the label triple, the update cannot change
  // any count (the reference's safe test, e.g.
  // ParaCOSM/CSM/matching/Parallel_SymBi/parrallel_symbi.cpp:3071-3127)
  bool Classify(uint v1, uint v2, uint label) override {
    csm_update u{'e', 1, 0, v1, v2, label};
    uint8_t safe = 0;
    check(csm_gpu_classify(ctx_, 1, &u, &safe));
    return safe != 0;
  }

  // Candidate-index size: set d1 / d2 flags over all query vertices
  // (the reference reports its hash-map sizes).
  void GetMemoryCost(size_t& num_edges, size_t& num_vertices) override {
    csm_stats s;
    check(csm_gpu_stats(ctx_, &s));
    num_edges = s.index_entries;
    num_vertices = s.index_vertices;
  }

  // A run of stream updates in one submit; the counters advance as if each
  // had been applied on its own, in order.  The data Graph is brought to the
  // state after the run.
  void ProcessUpdates(const std::vector<InsertUnit>& ups) {
    std::vector<csm_update> u(ups.size());
    for (size_t i = 0; i < ups.size(); i++)
      u[i] = csm_update{(uint8_t)ups[i].type, (uint8_t)(ups[i].is_add ? 1 : 0), 0, ups[i].id1, ups[i].id2,
                        ups[i].label};
    std::vector<csm_result> r(u.size());
    check(csm_gpu_submit(ctx_, u.size(), u.data()));
    check(csm_gpu_results(ctx_, seq_, u.size(), r.data()));
    if (print_enumeration_results_) print_matches();
    seq_ += u.size();
    for (size_t i = 0; i < ups.size(); i++) {
      num_positive_results_ += r[i].pos;
      num_negative_results_ += r[i].neg;
      const InsertUnit& x = ups[i];
      if (r[i].status == CSM_ST_INVALID) continue;
      if (x.type == 'v') { if (x.is_add) data_.AddVertex(x.id1, x.label); else data_.RemoveVertex(x.id1); }
      else if (x.is_add) data_.AddEdge(x.id1, x.id2, x.label);
      else data_.RemoveEdge(x.id1, x.id2);
    }
  }

  csm_ctx* context() const { return ctx_; }

 private:
  static constexpr uint32_t kEnumCapacity = 1u << 22;

  static void check(int rc) {
    if (rc != CSM_OK) {
      std::cout << "csm_gpu: " << csm_gpu_strerror(rc) << ": " << csm_gpu_last_error() << std::endl;
      exit(-1);
    }
  }

  // Vertex labels and undirected edges (each once, v < w) of a reference Graph.
  static void flatten(const Graph& g, std::vector<uint32_t>& vl, std::vector<uint32_t>& e) {
    const uint n = g.NumVertices();
    vl.resize(n);
    for (uint v = 0; v < n; v++) vl[v] = g.GetVertexLabel(v);
    for (uint v = 0; v < n; v++) {
      const std::vector<uint>& nb = g.GetNeighbors(v);
      const std::vector<uint>& lb = g.GetNeighborLabels(v);
      for (size_t i = 0; i < nb.size(); i++)
        if (v < nb[i]) { e.push_back(v); e.push_back(nb[i]); e.push_back(lb[i]); }
    }
  }

  void run_one(uint8_t type, uint8_t add, uint id1, uint id2, uint label) {
    csm_update u{type, add, 0, id1, id2, label};
    csm_result r;
    check(csm_gpu_submit(ctx_, 1, &u));
    check(csm_gpu_results(ctx_, seq_, 1, &r));
    if (print_enumeration_results_) print_matches();
    seq_++;
    num_positive_results_ += r.pos;
    num_negative_results_ += r.neg;
  }

  // Every embedding of the last submit, one "m0 m1 ... " line each.
  void print_matches() {
    const uint32_t nq = query_.NumVertices();
    uint64_t got = 0, found = 0;
    check(csm_gpu_matches(ctx_, nullptr, 0, &got, &found));
    if (found > kEnumCapacity) {
      std::cout << "csm_gpu: " << found << " embeddings found, at most " << kEnumCapacity << " kept" << std::endl;
      exit(-1);
    }
    std::vector<uint32_t> rec((size_t)(1 + nq) * (found ? found : 1));
    check(csm_gpu_matches(ctx_, rec.data(), found, &got, &found));
    for (uint64_t i = 0; i < got; i++) {
      const uint32_t* m = rec.data() + i * (1 + nq) + 1;
      for (uint32_t q = 0; q < nq; q++) std::cout << m[q] << " ";
      std::cout << "\n";
    }
  }

  csm_ctx* ctx_ = nullptr;
  uint64_t seq_ = 0;
};

#endif  // CSM_GPU_PLUGIN_H
