// Plugin classes over the C ABI (see plugins.h).
#include "plugins.h"

#include <algorithm>
#include <cstdio>

namespace csm {

matching::matching(const EdgeList& query, const EdgeList& data, size_t max_num_results, bool print_prep,
                   bool print_enum, bool homo, int algorithm, const GpuOptions& opt)
    : query_(query), data_(data), max_num_results_(max_num_results), print_preprocessing_results_(print_prep),
      print_enumeration_results_(print_enum), homomorphism_(homo), algo_(algorithm), opt_(opt) {
  csm_cfg cfg;
  csm_gpu_default_cfg(&cfg);
  cfg.algorithm = algorithm;
  cfg.homomorphism = homo ? 1 : 0;
  // the reference's "no cap" is UINT_MAX (main.cpp:681); the engine's is 0
  cfg.max_results = (max_num_results >= 0xffffffffull) ? 0 : (uint64_t)max_num_results;
  cfg.mode = opt.mode;
  cfg.max_batch = opt.max_batch;
  cfg.want_hash = opt.want_hash ? 1 : 0;
  cfg.device = opt.device;
  cfg.turboflux_compat = opt.turboflux_compat ? 1 : 0;
  cfg.warps_per_block = opt.warps_per_block;
  cfg.blocks_per_sm = opt.blocks_per_sm;
  cfg.vertex_headroom = opt.vertex_headroom;
  cfg.hbm_budget_bytes = opt.hbm_budget_bytes;
  cfg.deadline_ns = opt.deadline_ns;
  cfg.enum_capacity = opt.enum_capacity;
  cfg.graphs = opt.graphs ? CSM_GRAPHS_ON : CSM_GRAPHS_OFF;
  check(csm_gpu_create(&cfg, &ctx_));
}

matching::~matching() {
  for (csm_ctx* a : attached_) csm_gpu_destroy(a);
  if (ctx_) csm_gpu_destroy(ctx_);
}

int matching::check(int rc) {
  if (rc != CSM_OK && err_ == CSM_OK) {
    err_ = rc;
    const char* t = csm_gpu_last_error();
    err_text_ = t ? t : csm_gpu_strerror(rc);
  }
  return rc;
}

// BuildDAG + BuildDCS of the reference become: the query and the data graph
// are copied to the device, then the engine builds its plans and index.
void matching::Preprocessing() {
  if (err_) return;
  if (check(csm_gpu_set_query(ctx_, query_.n, query_.vlabels.data(), (uint32_t)query_.num_edges(),
                              query_.edges.data())))
    return;
  if (!opt_.more_queries.empty()) {  // every query's labels stay distinct in the shared graph
    std::vector<uint32_t> vl, el;
    for (const EdgeList& q : opt_.more_queries) {
      vl.insert(vl.end(), q.vlabels.begin(), q.vlabels.end());
      for (uint64_t i = 0; i < q.num_edges(); i++) el.push_back(q.edges[3 * i + 2]);
    }
    if (check(csm_gpu_reserve_labels(ctx_, (uint32_t)vl.size(), vl.data(), (uint32_t)el.size(), el.data()))) return;
  }
  if (check(csm_gpu_load_graph(ctx_, data_.n, data_.vlabels.data(), data_.num_edges(), data_.edges.data()))) return;
  if (check(csm_gpu_build_index(ctx_))) return;
  for (const EdgeList& q : opt_.more_queries) {
    csm_cfg c;
    csm_gpu_default_cfg(&c);
    c.algorithm = algo_;
    c.max_results = (max_num_results_ >= 0xffffffffull) ? 0 : (uint64_t)max_num_results_;
    c.want_hash = opt_.want_hash ? 1 : 0;
    c.warps_per_block = opt_.warps_per_block;
    c.blocks_per_sm = opt_.blocks_per_sm;
    csm_ctx* a = nullptr;
    if (check(csm_gpu_attach_query(ctx_, &c, q.n, q.vlabels.data(), (uint32_t)q.num_edges(), q.edges.data(), &a)))
      return;
    attached_.push_back(a);
  }
  if (print_preprocessing_results_ && !err_ && algo_ != CSM_ALGO_GRAPHFLOW) {
    csm_index_info info;
    if (!check(csm_gpu_index_info(ctx_, &info))) {
      // the reference's "DAG:" listing (SymBi/symbi.cpp:240-256)
      printf("DAG: \n");
      for (uint32_t i = 0; i < info.n_qv; i++) {
        const uint32_t u = info.order[i];
        printf("%u: (backwards: ", u);
        for (uint32_t p = 0; p < info.n_qv; p++)
          if ((info.parents[u] >> p) & 1u) printf("%u ", p);
        printf(") (forwards: ");
        for (uint32_t c = 0; c < info.n_qv; c++)
          if ((info.parents[c] >> u) & 1u) printf("%u ", c);
        printf(")\n");
      }
      printf("\n");
    }
  }
}

void matching::InitialMatching() {
  if (err_) return;
  uint64_t c = 0;
  if (!check(csm_gpu_initial_match(ctx_, &c))) num_initial_results_ += c;
  for (csm_ctx* a : attached_) {
    c = 0;
    if (check(csm_gpu_initial_match(a, &c))) return;
    num_initial_results_ += c;
  }
}

// Adds the attached queries' results for sequence numbers first .. first+n-1
// to out (counts summed, the largest status kept).
int matching::add_attached(uint64_t first, size_t n, csm_result* out) {
  if (attached_.empty()) return CSM_OK;
  std::vector<csm_result> r(n);
  for (csm_ctx* a : attached_) {
    if (check(csm_gpu_results(a, first, n, r.data()))) return err_;
    for (size_t i = 0; i < n; i++) {
      out[i].pos += r[i].pos;
      out[i].neg += r[i].neg;
      out[i].status = std::max(out[i].status, r[i].status);
    }
  }
  return CSM_OK;
}

void matching::run_one(const Update& u) {
  if (err_) return;
  csm_update cu;
  cu.type = u.type; cu.is_add = u.is_add; cu.pad = 0; cu.id1 = u.id1; cu.id2 = u.id2; cu.label = u.label;
  if (check(csm_gpu_submit(ctx_, 1, &cu))) return;
  const uint64_t first = seq_++;
  csm_result r;
  if (check(csm_gpu_results(ctx_, first, 1, &r))) return;
  if (add_attached(first, 1, &r)) return;
  num_positive_results_ += r.pos;
  num_negative_results_ += r.neg;
}

void matching::AddEdge(uint32_t v1, uint32_t v2, uint32_t label) { run_one(Update{'e', 1, 0, v1, v2, label}); }
void matching::RemoveEdge(uint32_t v1, uint32_t v2) { run_one(Update{'e', 0, 0, v1, v2, 0}); }
void matching::AddVertex(uint32_t id, uint32_t label) { run_one(Update{'v', 1, 0, id, 0, label}); }
void matching::RemoveVertex(uint32_t id) { run_one(Update{'v', 0, 0, id, 0, 0}); }

bool matching::Classify(uint32_t v1, uint32_t v2, uint32_t label) {
  csm_update cu{'e', 1, 0, v1, v2, label};
  uint8_t safe = 0;
  if (check(csm_gpu_classify(ctx_, 1, &cu, &safe))) return false;
  return safe != 0;
}

void matching::GetMemoryCost(size_t& num_edges, size_t& num_vertices) {
  csm_stats st;
  num_edges = num_vertices = 0;
  if (check(csm_gpu_stats(ctx_, &st))) return;
  num_edges = st.index_entries;
  num_vertices = st.index_vertices;
}

int matching::ProcessUpdates(const std::vector<Update>& ups, std::vector<csm_result>& out) {
  out.resize(ups.size());
  if (err_) return err_;
  if (ups.empty()) return CSM_OK;
  static_assert(sizeof(Update) == sizeof(csm_update), "update records share one layout");
  if (check(csm_gpu_submit(ctx_, ups.size(), reinterpret_cast<const csm_update*>(ups.data())))) return err_;
  const uint64_t first = seq_;
  seq_ += ups.size();
  if (check(csm_gpu_results(ctx_, first, ups.size(), out.data()))) return err_;
  if (add_attached(first, ups.size(), out.data())) return err_;
  for (const csm_result& r : out) {
    num_positive_results_ += r.pos;
    num_negative_results_ += r.neg;
  }
  return CSM_OK;
}

int matching::PrintMatches(size_t n) {
  if (err_) return err_;
  const uint32_t nq = query_.n;
  uint64_t kept = 0, found = 0;
  if (check(csm_gpu_matches(ctx_, nullptr, 0, &kept, &found))) return err_;  // sizes first
  std::vector<uint32_t> rec((size_t)std::min<uint64_t>(found, opt_.enum_capacity) * (1 + nq) + 1);
  if (check(csm_gpu_matches(ctx_, rec.data(), std::min<uint64_t>(found, opt_.enum_capacity), &kept, &found)))
    return err_;
  if (found > kept)
    fprintf(stderr, "print-enum: %llu embeddings found, %llu kept\n", (unsigned long long)found,
            (unsigned long long)kept);
  // group by update (counting sort on the leading word)
  std::vector<uint64_t> start(n + 1, 0);
  for (uint64_t r = 0; r < kept; r++) start[rec[r * (1 + nq)] + 1]++;
  for (size_t i = 0; i < n; i++) start[i + 1] += start[i];
  std::vector<uint64_t> order(kept), fill(start.begin(), start.end() - 1);
  for (uint64_t r = 0; r < kept; r++) order[fill[rec[r * (1 + nq)]]++] = r;
  std::string line;
  for (uint64_t r : order) {
    line.clear();
    for (uint32_t q = 0; q < nq; q++) { line += std::to_string(rec[r * (1 + nq) + 1 + q]); line += ' '; }
    puts(line.c_str());
  }
  return CSM_OK;
}

matching* make_plugin(const std::string& name, const EdgeList& q, const EdgeList& d, size_t max_results,
                      bool print_prep, bool print_enum, bool homo, const GpuOptions& opt) {
  if (name == "parallel_graphflow" || name == "graphflow")
    return new Parallel_Graphflow(q, d, max_results, print_prep, print_enum, homo, opt);
  if (name == "parallel_turboflux" || name == "turboflux")
    return new Parallel_TurboFlux(q, d, max_results, print_prep, print_enum, homo, opt);
  if (name == "parallel_symbi" || name == "symbi")
    return new Parrllel_SymBi(q, d, max_results, print_prep, print_enum, homo, opt);
  if (name == "parallel_calig" || name == "calig")
    return new Parallel_CaLiG(q, d, max_results, print_prep, print_enum, homo, opt);
  if (name == "parallel_newsp" || name == "newsp")
    return new CSMPP(q, d, max_results, print_prep, print_enum, homo, opt);
  return nullptr;
}

}  // namespace csm
