// C ABI of the engine: context, device memory, query plans, the per-batch
// launch sequence, results.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "csm_host.cuh"
#include "csm_index.cuh"
#include "csm_kernels.cuh"

namespace csm {

static thread_local std::string g_last_error;

int set_err(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CK(call)                                                                                      \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return set_err(CSM_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,       \
                                          cudaGetErrorString(e_));                                    \
  } while (0)

#define CKL()                                                                                         \
  do {                                                                                                \
    ctx->launches++;                                                                                  \
    cudaError_t e_ = cudaGetLastError();                                                              \
    if (e_ != cudaSuccess) return set_err(CSM_ECUDA, "%s:%d launch: %s", __FILE__, __LINE__,          \
                                          cudaGetErrorString(e_));                                    \
  } while (0)

static uint32_t ceil_log2(uint64_t x) {
  uint32_t b = 0;
  while ((1ULL << b) < x) b++;
  return b;
}

static inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)std::max<uint64_t>(1, (n + t - 1) / t); }

}  // namespace csm

using namespace csm;

struct csm_ctx {
  csm_cfg cfg;
  int dev = 0, sm_count = 0;
  cudaStream_t st = nullptr;
  DevMem mem;
  uint64_t launches = 0;
  // query
  bool has_query = false;
  uint32_t nq = 0;
  std::vector<uint32_t> qvl, qe;      // labels, (u, v, l) triples (deduplicated), as given
  std::vector<uint32_t> qlab_v, qlab_e;  // sorted distinct query labels (the label folding tables)
  std::vector<uint32_t> qvl_f;        // folded query vertex labels
  uint32_t* d_qlab = nullptr;
  std::vector<std::vector<uint32_t>> qnbr, qel;  // sorted adjacency
  Plan* h_plan = nullptr;
  Plan* d_plan = nullptr;
  size_t plan_bytes = 0;
  bool has_plan = false;
  // graph
  bool has_graph = false;
  DevGraph g{};
  std::vector<uint32_t> h_vlabel;  // folded vertex labels (kNone: no vertex), mirrored on the host
  // edge table (DevGraph::ekeys): upper bounds of its live keys and deleted
  // slots, from the updates submitted since it was last filled
  uint64_t e_live = 0, e_tomb = 0;
  uint64_t num_edges = 0;
  // candidate index
  IndexState index{};
  // batch buffers
  uint32_t bmax = 0, lcap = 0, task_cap = 0;
  csm_update* d_stream = nullptr; uint64_t stream_cap = 0;
  uint64_t *d_ukey = nullptr, *d_ukey2 = nullptr;
  uint32_t *d_useq = nullptr, *d_useq2 = nullptr;
  UpdInfo* d_info = nullptr;
  uint64_t *d_ins = nullptr, *d_ins2 = nullptr, *d_del = nullptr, *d_del2 = nullptr;
  uint64_t *d_tk = nullptr, *d_tk2 = nullptr, *d_ts = nullptr, *d_ts2 = nullptr;
  VRange *d_rins = nullptr, *d_rdel = nullptr, *d_rt = nullptr;
  uint32_t* d_ins_dst = nullptr;
  unsigned int* d_cnt = nullptr;  // [0] n_ins [1] n_del [2] n_t [3] n_rins [4] n_rdel [5] n_rt [6] n_tasks [7] task_next
  Task* d_tasks = nullptr;
  unsigned long long *d_count = nullptr, *d_hash = nullptr, *d_bytes = nullptr;
  unsigned int* d_stop = nullptr;
  uint32_t* d_safe = nullptr;
  unsigned long long* d_stamp = nullptr;  // [0] submit time (globaltimer)
  SearchQueue* d_q = nullptr;
  DTask* d_dq = nullptr;
  unsigned long long* d_qseq = nullptr;
  uint32_t qcap = 0;
  SearchStats* d_sstat = nullptr;
  csm_result* d_results = nullptr; uint64_t results_cap = 0;
  void* d_cub = nullptr; size_t cub_bytes = 0;
  // bookkeeping
  uint64_t seq_next = 0, last_first = 0, last_n = 0;
  uint64_t updates_done = 0, v_updates = 0, e_updates = 0, batches = 0;
  uint64_t tot_pos = 0, tot_neg = 0, tot_unsafe = 0;
  bool totals_dirty = false;
  std::vector<csm_result> h_last;  // host copy of the last submit's results (filled lazily)
  bool h_last_valid = false;
  cudaEvent_t ev_start = nullptr, ev_end = nullptr;
  double last_ms = 0, total_ms = 0;
  // CUDA events around every search launch of the pending submit
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> sev;
  size_t sev_used = 0;
  uint64_t search_launches = 0, work_bytes = 0;
  double search_ms = 0;
  // standing queries sharing one data graph: the owner holds the graph and
  // applies mutations; attached contexts hold a query, its plan and index
  csm_ctx* owner = nullptr;
  std::vector<csm_ctx*> attached;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // CUDA-graph replay of the batch launch sequence (owner only): one graph
  // per batch size, rebuilt when the query set, the vertex count or the
  // launch shape changes.  Batches read their updates from d_gups and write
  // results to d_gres (one staging array per query), copied out after replay.
  struct GraphEntry {
    uint32_t B;
    uint64_t version;
    cudaGraphExec_t exec;
    std::vector<uint64_t> launches;  // per query (owner, then attached)
  };
  std::vector<GraphEntry> graphs;
  uint64_t graph_version = 1, graph_replays = 0;
  bool capturing = false;
  csm_update* d_gups = nullptr;
  csm_result* d_gres = nullptr;
  csm_update* d_gpad = nullptr;  // padding records: self loops, which are invalid and change nothing
  // match-set output of the last submit (cfg.enum_capacity > 0)
  uint32_t* d_enum = nullptr;
  unsigned long long* d_enum_n = nullptr;
};

namespace csm {

// ------------------------------------------------------------------ plans

// GraphFlow matching orders (ParaCOSM/CSM/matching/GraphFlow/graphflow.cpp:36-169):
// order 0 starts at the max-degree query vertex; order i > 0 starts at the
// i-th backward edge of order 0; every next vertex maximises the number of
// already ordered neighbours, ties broken by larger degree, then smaller id.
static void graphflow_orders(const csm_ctx* ctx, std::vector<std::vector<uint32_t>>& order) {
  const uint32_t n = ctx->nq, m = (uint32_t)(ctx->qe.size() / 3);
  order.assign(m, std::vector<uint32_t>(n, 0));
  std::vector<uint32_t> offs(n, 0), csr(m + 1, 0);
  auto deg = [&](uint32_t u) { return (uint32_t)ctx->qnbr[u].size(); };
  auto pick = [&](std::vector<char>& vis) {
    uint32_t best = kNone, best_adj = 0;
    for (uint32_t j = 0; j < n; j++) {
      if (vis[j]) continue;
      uint32_t adj = 0;
      for (uint32_t o : ctx->qnbr[j]) if (vis[o]) adj++;
      if (!adj) continue;
      if (best == kNone || (adj == best_adj && deg(j) > deg(best)) || adj > best_adj) { best_adj = adj; best = j; }
    }
    return best;
  };
  std::vector<char> vis(n, 0);
  uint32_t maxd = 0;
  for (uint32_t i = 0; i < n; i++) if (deg(i) > maxd) { maxd = deg(i); order[0][0] = i; }
  vis[order[0][0]] = 1;
  for (uint32_t i = 1; i < n; i++) {
    const uint32_t u = pick(vis);
    order[0][i] = u; vis[u] = 1;
    offs[i] = offs[i - 1];
    for (uint32_t o : ctx->qnbr[u]) if (vis[o]) csr[offs[i]++] = o;
  }
  for (uint32_t i = 1; i < m; i++) {
    std::vector<char> v2(n, 0);
    const uint32_t p = (uint32_t)(std::lower_bound(offs.begin(), offs.end(), i + 1) - offs.begin());
    order[i][0] = order[0][p];
    order[i][1] = csr[i];
    v2[order[i][0]] = 1; v2[order[i][1]] = 1;
    for (uint32_t j = 2; j < n; j++) { const uint32_t u = pick(v2); order[i][j] = u; v2[u] = 1; }
  }
}

static uint32_t fold_host(const std::vector<uint32_t>& sorted, uint32_t l) {
  auto it = std::lower_bound(sorted.begin(), sorted.end(), l);
  return (it != sorted.end() && *it == l) ? (uint32_t)(it - sorted.begin()) : (uint32_t)sorted.size();
}

// Folded label of query edge (a, b), or kNone if a and b are not adjacent.
static uint32_t qedge_label(const csm_ctx* ctx, uint32_t a, uint32_t b) {
  const auto& nb = ctx->qnbr[a];
  auto it = std::lower_bound(nb.begin(), nb.end(), b);
  if (it == nb.end() || *it != b) return kNone;
  return fold_host(ctx->qlab_e, ctx->qel[a][(size_t)(it - nb.begin())]);
}

// Independent tail of order o (PlanAnchor): the longest suffix o[s..n-1],
// s >= 2, with no query edge inside and no vertex label more than kTailGroup
// times; used when it has at least two vertices.
static void plan_tail(const csm_ctx* ctx, const std::vector<uint32_t>& o, PlanAnchor& A) {
  const uint32_t n = ctx->nq;
  A.tail_at = 0; A.n_groups = 0; A.prefix_mask = 0xffffffffu;
  if (n < 4) return;
  std::vector<int> pos(n);
  for (uint32_t i = 0; i < n; i++) pos[o[i]] = (int)i;
  uint32_t s = n - 1;
  while (s > 2) {
    const uint32_t u = o[s - 1];
    bool stop = false;
    for (uint32_t w : ctx->qnbr[u]) if (pos[w] >= (int)s) stop = true;
    uint32_t same = 0;
    for (uint32_t i = s; i < n; i++) same += ctx->qvl_f[o[i]] == ctx->qvl_f[u];
    if (stop || same >= kTailGroup) break;
    s--;
  }
  if (n - s < 2) return;
  A.tail_at = (uint8_t)(s - 1);
  A.prefix_mask = (1u << s) - 1u;
  std::vector<char> done(n, 0);
  uint32_t k = 0;
  for (uint32_t d = s; d < n; d++) {
    if (done[d]) continue;
    uint32_t g = 0;
    for (uint32_t e = d; e < n; e++)
      if (!done[e] && ctx->qvl_f[o[e]] == ctx->qvl_f[o[d]]) { done[e] = 1; A.gpos[k++] = (uint8_t)e; g++; }
    A.gsize[A.n_groups++] = (uint8_t)g;
  }
}

static int build_plan(csm_ctx* ctx) {
  std::vector<std::vector<uint32_t>> order;
  graphflow_orders(ctx, order);
  Plan* P = ctx->h_plan;
  memset(P, 0, sizeof(Plan));
  P->n = ctx->nq;
  P->n_anchor = (uint32_t)order.size();
  const uint32_t n_el = ctx->g.n_el;
  for (uint32_t a = 0; a < P->n_anchor; a++) {
    PlanAnchor& A = P->anchors[a];
    const auto& o = order[a];
    A.la = ctx->qvl_f[o[0]]; A.lb = ctx->qvl_f[o[1]]; A.el = qedge_label(ctx, o[0], o[1]);
    uint32_t nb_total = 0;
    for (uint32_t d = 0; d < ctx->nq; d++) {
      PlanPos& pp = A.pos[d];
      pp.qv = (uint8_t)o[d];
      pp.nb = 0; pp.boff = (uint16_t)nb_total; pp.samelab = 0;
      if (d < 2) continue;
      for (uint32_t j = 0; j < d; j++) {
        if (ctx->qvl_f[o[j]] == ctx->qvl_f[o[d]]) pp.samelab |= 1u << j;
        const uint32_t l = qedge_label(ctx, o[d], o[j]);
        if (l == kNone) continue;
        if (nb_total >= kMaxQE || pp.nb >= kMaxBack) return set_err(CSM_EUNSUPPORTED, "query too dense");
        A.back_pos[nb_total] = (uint8_t)j;
        A.back_combo[nb_total] = (uint16_t)(ctx->qvl_f[o[d]] * n_el + l);
        nb_total++; pp.nb++;
      }
      if (pp.nb == 0) return set_err(CSM_EINVAL, "query graph is not connected");
    }
    plan_tail(ctx, o, A);
  }
  ctx->plan_bytes = offsetof(Plan, anchors) + (size_t)P->n_anchor * sizeof(PlanAnchor);
  if (!ctx->d_plan) {
    int rc = ctx->mem.alloc((void**)&ctx->d_plan, sizeof(Plan));
    if (rc) return rc;
  }
  CK(cudaMemcpyAsync(ctx->d_plan, P, ctx->plan_bytes, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->has_plan = true;
  return CSM_OK;
}

// --------------------------------------------------------- batch buffers

static int ensure_batch_buffers(csm_ctx* ctx) {
  if (ctx->d_ukey) return CSM_OK;
  const uint32_t B = ctx->bmax;
  const uint32_t L = 4 * B + 64;
  ctx->lcap = L;
  const uint32_t na = std::max<uint32_t>(1, (uint32_t)(ctx->qe.size() / 3));
  ctx->task_cap = B * 2 * na;
  DevMem& m = ctx->mem;
  int rc = 0;
#define AL(p, sz) do { rc = m.alloc((void**)&(p), (sz)); if (rc) return rc; } while (0)
  AL(ctx->d_ukey, 8ull * B); AL(ctx->d_ukey2, 8ull * B);
  AL(ctx->d_useq, 4ull * B); AL(ctx->d_useq2, 4ull * B);
  AL(ctx->d_info, sizeof(UpdInfo) * (size_t)B);
  AL(ctx->d_ins, 8ull * L); AL(ctx->d_ins2, 8ull * L);
  AL(ctx->d_del, 8ull * L); AL(ctx->d_del2, 8ull * L);
  AL(ctx->d_tk, 8ull * L); AL(ctx->d_tk2, 8ull * L);
  AL(ctx->d_ts, 8ull * L); AL(ctx->d_ts2, 8ull * L);
  AL(ctx->d_rins, sizeof(VRange) * (size_t)L); AL(ctx->d_rdel, sizeof(VRange) * (size_t)L);
  AL(ctx->d_rt, sizeof(VRange) * (size_t)L);
  AL(ctx->d_ins_dst, 4ull * L);
  AL(ctx->d_cnt, 64);
  AL(ctx->d_tasks, sizeof(Task) * (size_t)ctx->task_cap);
  AL(ctx->d_count, 8ull * B); AL(ctx->d_hash, 8ull * B); AL(ctx->d_bytes, 8ull * B);
  AL(ctx->d_stop, 4ull * B); AL(ctx->d_safe, 4ull * B);
  AL(ctx->d_stamp, 64);
  AL(ctx->d_gups, sizeof(csm_update) * (size_t)B);
  AL(ctx->d_gres, sizeof(csm_result) * (size_t)B);
  AL(ctx->d_gpad, sizeof(csm_update) * (size_t)B);
  if (ctx->cfg.enum_capacity) {
    AL(ctx->d_enum, 4ull * (1 + ctx->nq) * ctx->cfg.enum_capacity);
    AL(ctx->d_enum_n, 16);
    CK(cudaMemsetAsync(ctx->d_enum_n, 0, 16, ctx->st));
  }
  {
    std::vector<csm_update> pad(B, csm_update{'e', 1, 0, 0, 0, 0});
    CK(cudaMemcpyAsync(ctx->d_gpad, pad.data(), sizeof(csm_update) * (size_t)B, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  ctx->qcap = 1u << 16;  // outstanding handed-over tasks never exceed the idle warps
  AL(ctx->d_q, sizeof(SearchQueue));
  AL(ctx->d_sstat, sizeof(SearchStats));
  CK(cudaMemsetAsync(ctx->d_sstat, 0, sizeof(SearchStats), ctx->st));
  AL(ctx->d_dq, sizeof(DTask) * (size_t)ctx->qcap);
  AL(ctx->d_qseq, 8ull * ctx->qcap);
  CK(cudaMemsetAsync(ctx->d_q, 0, sizeof(SearchQueue), ctx->st));
  {
    std::vector<unsigned long long> seq(ctx->qcap);
    for (uint32_t i = 0; i < ctx->qcap; i++) seq[i] = i;
    CK(cudaMemcpyAsync(ctx->d_qseq, seq.data(), 8ull * ctx->qcap, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
#undef AL
  // CUB scratch: the largest of the sorts issued per batch
  size_t b1 = 0, b2 = 0, b3 = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, b1, ctx->d_ukey, ctx->d_ukey2, ctx->d_useq, ctx->d_useq2, (int)B, 0, 64, ctx->st));
  CK(cub::DeviceRadixSort::SortKeys(nullptr, b2, ctx->d_ins, ctx->d_ins2, (int)L, 0, 64, ctx->st));
  CK(cub::DeviceRadixSort::SortPairs(nullptr, b3, ctx->d_tk, ctx->d_tk2, ctx->d_ts, ctx->d_ts2, (int)L, 0, 64, ctx->st));
  const size_t need = std::max(b1, std::max(b2, b3));
  if (need > ctx->cub_bytes) {
    if (ctx->d_cub) ctx->mem.release(ctx->d_cub, ctx->cub_bytes);
    ctx->d_cub = nullptr;
    rc = ctx->mem.alloc(&ctx->d_cub, need);
    if (rc) return rc;
    ctx->cub_bytes = need;
  }
  return CSM_OK;
}

static int ensure_results(csm_ctx* ctx, uint64_t n) {
  if (n <= ctx->results_cap) return CSM_OK;
  if (ctx->d_results) ctx->mem.release(ctx->d_results, ctx->results_cap * sizeof(csm_result));
  ctx->d_results = nullptr;
  uint64_t cap = std::max<uint64_t>(n, 1024);
  int rc = ctx->mem.alloc((void**)&ctx->d_results, cap * sizeof(csm_result));
  if (rc) return rc;
  ctx->results_cap = cap;
  return CSM_OK;
}

static int ensure_stream(csm_ctx* ctx, uint64_t n) {
  if (n <= ctx->stream_cap) return CSM_OK;
  if (ctx->d_stream) ctx->mem.release(ctx->d_stream, ctx->stream_cap * sizeof(csm_update));
  ctx->d_stream = nullptr;
  uint64_t cap = std::max<uint64_t>(n, 1024);
  int rc = ctx->mem.alloc((void**)&ctx->d_stream, cap * sizeof(csm_update));
  if (rc) return rc;
  ctx->stream_cap = cap;
  return CSM_OK;
}

__global__ void k_stamp(unsigned long long* stamp) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  stamp[0] = t;
}

// ------------------------------------------------------------ batches
//
// One batch of B edge updates runs in phases.  The context that owns the
// data graph applies the insertions (the union graph), every standing query
// -- the owner's and those attached to it, each on its own stream -- brings
// its index to the union graph and searches, then the owner applies the
// deletions and every query brings its index to the graph after the batch.
// Events order the streams; the searches of different queries overlap.

// Owner: group the batch's updates per edge, resolve each edge's timeline,
// temporal entries, CSR -> union graph.
static int batch_mutate_insert(csm_ctx* ctx, const csm_update* ups, uint32_t B, uint32_t L) {
  cudaStream_t st = ctx->st;
  DevGraph& g = ctx->g;
  const KeyBits kb = g.kb;
  CK(cudaMemsetAsync(ctx->d_cnt, 0, 64, st));
  CK(cudaMemsetAsync(ctx->d_ins, 0xff, 8ull * L, st));
  CK(cudaMemsetAsync(ctx->d_del, 0xff, 8ull * L, st));
  CK(cudaMemsetAsync(ctx->d_tk, 0xff, 8ull * L, st));
  unsigned int* c = ctx->d_cnt;
  k_batch_init<<<blocks_for(B, 256), 256, 0, st>>>(ups, B, g, ctx->d_ukey, ctx->d_useq, ctx->d_info); CKL();
  size_t tb = ctx->cub_bytes;
  CK(cub::DeviceRadixSort::SortPairs(ctx->d_cub, tb, ctx->d_ukey, ctx->d_ukey2, ctx->d_useq, ctx->d_useq2, (int)B, 0, 64, st));
  ResolveOut ro{ctx->d_ins, c + 0, ctx->d_del, c + 1, ctx->d_tk, ctx->d_ts, c + 2, L};
  k_resolve<<<blocks_for(B, 128), 128, 0, st>>>(ctx->d_ukey2, ctx->d_useq2, B, g, ups, ctx->d_info, ro); CKL();
  const int end_bit = (int)kb.total();
  tb = ctx->cub_bytes;
  CK(cub::DeviceRadixSort::SortKeys(ctx->d_cub, tb, ctx->d_ins, ctx->d_ins2, (int)L, 0, end_bit, st));
  tb = ctx->cub_bytes;
  CK(cub::DeviceRadixSort::SortKeys(ctx->d_cub, tb, ctx->d_del, ctx->d_del2, (int)L, 0, end_bit, st));
  tb = ctx->cub_bytes;
  CK(cub::DeviceRadixSort::SortPairs(ctx->d_cub, tb, ctx->d_tk, ctx->d_tk2, ctx->d_ts, ctx->d_ts2, (int)L, 0, end_bit, st));
  k_ranges<<<blocks_for(L, 256), 256, 0, st>>>(ctx->d_ins2, L, kb, ctx->d_rins, c + 3, g.dir, g.nc); CKL();
  k_ranges<<<blocks_for(L, 256), 256, 0, st>>>(ctx->d_del2, L, kb, ctx->d_rdel, c + 4, g.dir, g.nc); CKL();
  k_ranges<<<blocks_for(L, 256), 256, 0, st>>>(ctx->d_tk2, L, kb, ctx->d_rt, c + 5, g.dir, g.nc); CKL();
  g.t_key = ctx->d_tk2;
  g.t_span = reinterpret_cast<int2*>(ctx->d_ts2);
  k_temporal_set<<<blocks_for(L, 256), 256, 0, st>>>(ctx->d_rt, c + 5, g); CKL();
  // CSR -> union graph (relocating rows, and compacting the pools first if needed)
  k_reloc_need<<<blocks_for(L, 256), 256, 0, st>>>(ctx->d_rins, c + 3, g); CKL();
  k_compact_check<<<1, 1, 0, st>>>(g); CKL();
  k_compact_copy<<<ctx->sm_count * 4, 1024, 0, st>>>(g); CKL();
  k_compact_finish<<<1, 1, 0, st>>>(g); CKL();
  const uint32_t mut_blocks = std::min<uint32_t>(blocks_for(L * 32ull, 256), (uint32_t)ctx->sm_count * 16);
  launch_mut_insert(ctx->d_rins, c + 3, ctx->d_ins2, ctx->d_ins_dst, g, mut_blocks, (uint32_t)ctx->sm_count * 2, st);
  CKL();
  ctx->launches++;
  if (g.emask) { k_edge_list<<<blocks_for(L, 256), 256, 0, st>>>(ctx->d_ins2, L, g, 0u); CKL(); }
  return CSM_OK;
}

// Launch shape of the search: the configured (or autotuned) one, else 8
// warps per block and as many blocks per SM as can be resident.
static void search_shape(const csm_ctx* q, uint32_t& warps, uint32_t& bps) {
  warps = q->cfg.warps_per_block ? q->cfg.warps_per_block : 8;
  if (warps != 4 && warps != 8 && warps != 16) warps = 8;
  bps = q->cfg.blocks_per_sm ? q->cfg.blocks_per_sm : 0;
  if (!bps) {
    const int mode = q->d_enum ? 1 : ((!q->cfg.want_hash && !q->cfg.tail_enumerate) ? 2 : 0);
    bps = std::max<uint32_t>(1, search_max_blocks(q->nq, warps, mode));
  }
}

static int query_seed_search(csm_ctx* q, csm_ctx* o, uint32_t B, csm_result* out);

// One standing query q over the owner o's union graph: index to the union
// graph, seeds, search, per-update results; on q's stream.
static int batch_query_search(csm_ctx* q, csm_ctx* o, uint32_t B, uint32_t L, csm_result* out) {
  csm_ctx* ctx = q;  // launches are counted on the query's context
  cudaStream_t st = q->st;
  const DevGraph& g = o->g;
  CK(cudaMemsetAsync(q->d_count, 0, 8ull * B, st));
  CK(cudaMemsetAsync(q->d_bytes, 0, 8ull * B, st));
  CK(cudaMemsetAsync(q->d_stop, 0, 4ull * B, st));
  if (q->cfg.want_hash) CK(cudaMemsetAsync(q->d_hash, 0, 8ull * B, st));
  unsigned int* c = q->d_cnt;
  if (q != o) CK(cudaMemsetAsync(c, 0, 64, st));
  int rc = index_apply_edges(q->index, g, o->d_ins2, L, st, &q->launches);
  if (rc) return rc;
  return query_seed_search(q, o, B, out);
}

// Seeds, search and per-update results of query q over the owner o's graph
// for the B updates described by o->d_info (the counters were cleared).
static int query_seed_search(csm_ctx* q, csm_ctx* o, uint32_t B, csm_result* out) {
  csm_ctx* ctx = q;  // launches are counted on the query's context
  cudaStream_t st = q->st;
  const DevGraph& g = o->g;
  unsigned int* c = q->d_cnt;
  k_seed<<<blocks_for(B, 128), 128, 0, st>>>(B, o->d_info, g, q->d_plan, q->index.d2, q->index.words,
                                              q->d_tasks, c + 6, q->task_cap, q->d_safe, &g.ps->error,
                                              q->cfg.shard_rank, q->cfg.shard_count,
                                              (uint32_t)q->cfg.turboflux_compat,
                                              q->cfg.algorithm == CSM_ALGO_CALIG ? 1u : 0u); CKL();
  SearchParams sp{};
  sp.g = g; sp.plan = q->d_plan; sp.tasks = q->d_tasks; sp.n_tasks = c + 6; sp.task_cap = q->task_cap;
  sp.task_next = c + 7; sp.info = o->d_info; sp.count = q->d_count; sp.hash = q->d_hash; sp.bytes = q->d_bytes;
  sp.stop = q->d_stop;
  sp.d2 = q->index.d2; sp.d2_words = q->index.words; sp.cap = q->cfg.max_results;
  sp.homo = q->cfg.homomorphism; sp.want_hash = q->cfg.want_hash; sp.error = &g.ps->error;
  sp.q = q->d_q; sp.dq = q->d_dq; sp.qseq = q->d_qseq; sp.qcap = q->qcap;
  sp.wait_limit_ns = 30ull * 1000000000ull;
  sp.slot_limit_ns = 100ull * 1000000ull;
  sp.task_limit_ns = 20ull * 1000000000ull;
  sp.batch = B;
  sp.sstat = q->d_sstat;
  sp.deadline_ns = q->cfg.deadline_ns;
  sp.donate_every = q->cfg.donate_every;
  sp.split_deep = q->cfg.split_deep;
  sp.tail = (!q->cfg.want_hash && !q->d_enum && !q->cfg.tail_enumerate) ? 1u : 0u;
  if (q->d_enum) {
    sp.enum_buf = q->d_enum; sp.enum_n = q->d_enum_n; sp.enum_cap = q->cfg.enum_capacity;
    sp.enum_base = (uint32_t)(out - q->d_results);  // this batch's first update within the submit
    sp.enum_stride = 1 + q->nq;
  }
  uint32_t warps, bps;
  search_shape(q, warps, bps);
  if (o->capturing) {  // replays are not timed per search
    launch_search(sp, q->nq, (uint32_t)q->sm_count * bps, warps, st); CKL();
  } else {
    if (q->sev_used == q->sev.size()) {
      cudaEvent_t a, b;
      CK(cudaEventCreate(&a));
      CK(cudaEventCreate(&b));
      q->sev.emplace_back(a, b);
    }
    CK(cudaEventRecord(q->sev[q->sev_used].first, st));
    launch_search(sp, q->nq, (uint32_t)q->sm_count * bps, warps, st); CKL();
    CK(cudaEventRecord(q->sev[q->sev_used].second, st));
    q->sev_used++;
  }
  k_finalize<<<blocks_for(B, 256), 256, 0, st>>>(B, o->d_info, q->d_count, q->d_hash, q->d_bytes,
                                                  q->d_safe, q->d_stop, q->cfg.max_results, q->cfg.want_hash,
                                                  out, (q->cfg.shard_count > 1 && q->cfg.shard_rank) ? 0u : 16u,
                                                  o->d_stamp);
  CKL();
  return CSM_OK;
}

// Stream `waiter` continues after the work queued so far on `signaller`.
static int stream_after(cudaStream_t waiter, cudaStream_t signaller, cudaEvent_t ev) {
  CK(cudaEventRecord(ev, signaller));
  CK(cudaStreamWaitEvent(waiter, ev, 0));
  return CSM_OK;
}

// Launch sequence of one batch of B edge updates already in device memory;
// out_q[k] is the result array of attached query k (in ctx->attached order).
static int run_edge_batch(csm_ctx* ctx, const csm_update* ups, uint32_t B, csm_result* out,
                          const std::vector<csm_result*>& out_q) {
  cudaStream_t st = ctx->st;
  const uint32_t L = std::min<uint32_t>(ctx->lcap, 4 * B + 64);
  int rc = batch_mutate_insert(ctx, ups, B, L);
  if (rc) return rc;
  // every query: index to the union graph, then search
  for (size_t k = 0; k < ctx->attached.size(); k++) {
    csm_ctx* a = ctx->attached[k];
    a->g = ctx->g;
    rc = stream_after(a->st, st, ctx->ev_fork);
    if (!rc) rc = batch_query_search(a, ctx, B, L, out_q[k]);
    if (rc) return rc;
  }
  rc = batch_query_search(ctx, ctx, B, L, out);
  if (rc) return rc;
  for (csm_ctx* a : ctx->attached) {
    rc = stream_after(st, a->st, a->ev_join);
    if (rc) return rc;
  }
  // union graph -> CSR after the batch, and every index to it
  unsigned int* c = ctx->d_cnt;
  DevGraph& g = ctx->g;
  const uint32_t mut_blocks = std::min<uint32_t>(blocks_for(L * 32ull, 256), (uint32_t)ctx->sm_count * 16);
  launch_mut_delete(ctx->d_rdel, c + 4, ctx->d_del2, ctx->d_ins_dst, g, mut_blocks, (uint32_t)ctx->sm_count * 2, st);
  CKL();
  ctx->launches++;
  if (g.emask) { k_edge_list<<<blocks_for(L, 256), 256, 0, st>>>(ctx->d_del2, L, g, 1u); CKL(); }
  for (csm_ctx* a : ctx->attached) {
    rc = stream_after(a->st, st, ctx->ev_fork);
    if (!rc) rc = index_apply_edges(a->index, g, ctx->d_del2, L, a->st, &a->launches);
    if (rc) return rc;
  }
  for (csm_ctx* a : ctx->attached) {
    rc = stream_after(st, a->st, a->ev_join);
    if (rc) return rc;
  }
  rc = index_apply_edges(ctx->index, g, ctx->d_del2, L, st, &ctx->launches);
  if (rc) return rc;
  k_temporal_clear<<<blocks_for(L, 256), 256, 0, st>>>(ctx->d_rt, c + 5, g); CKL();
  ctx->batches++;
  for (csm_ctx* a : ctx->attached) a->batches++;
  return CSM_OK;
}

// ------------------------------------------------- one update per launch
//
// The plain form (CSM_MODE_PLAIN) runs each edge update as its own short
// launch sequence.  An edge whose label triple (L(v1), L(v2), label) matches
// no query edge can neither be part of an embedding nor change a candidate
// index (every index condition counts only edges whose label triple matches
// a query edge), so such an update mutates the graph and reports zero; the
// host decides this from its mirror of the vertex labels.  A deletion counts
// with the edge's own label, which the host does not know, so a deletion is
// only decided this way when no query edge has its vertex-label pair.
// Launches per update:
//   no matching query edge: resolve, [compaction copy,] mutate        2-3
//   insertion:  resolve, compaction copy, mutate, index marks + round,
//               seeds, search queue + search, results                 9
//   deletion:   resolve, seeds, search queue + search, results,
//               mutate, index marks + round                           8
// (the compaction copy returns at once unless the insertion's relocation
// does not fit; GraphFlow has no index rounds).

// True when some query edge may match the update's label triple.
static bool plain_may_count(const csm_ctx* ctx, const csm_update& u) {
  const DevGraph& g = ctx->g;
  if (u.type != 'e' || u.id1 >= g.n || u.id2 >= g.n || u.id1 == u.id2) return false;  // INVALID
  const uint32_t L1 = ctx->h_vlabel[u.id1], L2 = ctx->h_vlabel[u.id2];
  if (L1 == kNone || L2 == kNone) return false;
  const uint32_t el = fold_host(ctx->qlab_e, u.label);
  const Plan* P = ctx->h_plan;
  for (uint32_t a = 0; a < P->n_anchor; a++) {
    const PlanAnchor& A = P->anchors[a];
    if (u.is_add && A.el != el) continue;
    if ((A.la == L1 && A.lb == L2) || (A.la == L2 && A.lb == L1)) return true;
  }
  return false;
}

// One edge update of the plain form (no attached queries); d_up is the record
// in device memory, h its host copy.
static int run_plain_edge(csm_ctx* ctx, const csm_update* d_up, const csm_update& h, csm_result* out) {
  cudaStream_t st = ctx->st;
  const DevGraph& g = ctx->g;
  uint64_t* keys = ctx->d_ins2;
  k_plain_resolve<<<1, 32, 0, st>>>(d_up, g, ctx->d_info, keys, ctx->d_cnt, ctx->d_count, ctx->d_hash, ctx->d_bytes,
                                     ctx->d_stop);
  CKL();
  if (h.type == 'e' && h.is_add) {
    k_compact_copy<<<ctx->sm_count * 4, 1024, 0, st>>>(g);  // returns at once unless the pool must be compacted
    CKL();
  }
  int rc = CSM_OK;
  if (!plain_may_count(ctx, h)) {
    k_plain_mutate<<<1, 256, 0, st>>>(g, ctx->d_info, keys, out, ctx->d_stamp, 16u);
    CKL();
  } else if (h.is_add) {
    k_plain_mutate<<<1, 256, 0, st>>>(g, ctx->d_info, keys, nullptr, nullptr, 16u);
    CKL();
    rc = index_apply_edge_one(ctx->index, g, keys, st, &ctx->launches);
    if (!rc) rc = query_seed_search(ctx, ctx, 1, out);
  } else {
    rc = query_seed_search(ctx, ctx, 1, out);
    if (rc) return rc;
    k_plain_mutate<<<1, 256, 0, st>>>(g, ctx->d_info, keys, nullptr, nullptr, 16u);
    CKL();
    rc = index_apply_edge_one(ctx->index, g, keys, st, &ctx->launches);
  }
  if (rc) return rc;
  ctx->batches++;
  return CSM_OK;
}

// Vertex deletion (Graph::RemoveVertex, ParaCOSM/CSM/graph/graph.cpp:51-56, and
// the plugins' RemoveVertex, e.g. SymBi/symbi.cpp:992-1021): every incident
// edge leaves both endpoint rows, every query's index follows, then the slot
// loses its label.  No embeddings are counted, as in the reference.
static int run_vertex_delete(csm_ctx* ctx, uint32_t v) {
  cudaStream_t st = ctx->st;
  DevGraph& g = ctx->g;
  uint32_t deg = 0;
  CK(cudaMemcpyAsync(&deg, g.dir + (size_t)v * (g.nc + 1) + g.nc, 4, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  std::vector<csm_ctx*> all{ctx};
  all.insert(all.end(), ctx->attached.begin(), ctx->attached.end());
  if (deg) {
    const uint32_t K = 2 * deg;
    uint64_t *keys = nullptr, *keys2 = nullptr;
    VRange* ranges = nullptr;
    unsigned int* nr = nullptr;
    void* tmp = nullptr;
    size_t tb = 0;
    CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys, keys2, (int)K, 0, (int)g.kb.total(), st));
    int rc = ctx->mem.alloc((void**)&keys, 8ull * K);
    if (!rc) rc = ctx->mem.alloc((void**)&keys2, 8ull * K);
    if (!rc) rc = ctx->mem.alloc((void**)&ranges, sizeof(VRange) * (size_t)K);
    if (!rc) rc = ctx->mem.alloc((void**)&nr, 16);
    if (!rc) rc = ctx->mem.alloc(&tmp, tb);
    auto release = [&]() {
      ctx->mem.release(keys, 8ull * K); ctx->mem.release(keys2, 8ull * K);
      ctx->mem.release(ranges, sizeof(VRange) * (size_t)K); ctx->mem.release(nr, 16); ctx->mem.release(tmp, tb);
    };
    if (rc) { release(); return rc; }
    k_vdel_keys<<<blocks_for(deg, 256), 256, 0, st>>>(g, v, deg, keys); CKL();
    CK(cub::DeviceRadixSort::SortKeys(tmp, tb, keys, keys2, (int)K, 0, (int)g.kb.total(), st));
    CK(cudaMemsetAsync(nr, 0, 16, st));
    k_ranges<<<blocks_for(K, 256), 256, 0, st>>>(keys2, K, g.kb, ranges, nr, g.dir, g.nc); CKL();
    const uint32_t mut_blocks = std::min<uint32_t>(blocks_for(K * 32ull, 256), (uint32_t)ctx->sm_count * 16);
    launch_mut_delete(ranges, nr, keys2, reinterpret_cast<uint32_t*>(keys), g, mut_blocks, (uint32_t)ctx->sm_count * 2,
                      st);
    CKL();
    ctx->launches++;
    if (g.emask) { k_edge_list<<<blocks_for(K, 256), 256, 0, st>>>(keys2, K, g, 1u); CKL(); }
    ctx->e_tomb += deg;
    for (csm_ctx* q : all) {
      if (q != ctx) { q->g = g; rc = stream_after(q->st, st, ctx->ev_fork); }
      if (!rc) rc = index_apply_edges(q->index, g, keys2, K, q->st, &q->launches);
      if (!rc && q != ctx) rc = stream_after(st, q->st, q->ev_join);
      if (rc) { release(); return rc; }
    }
    CK(cudaStreamSynchronize(st));
    release();
  }
  CK(cudaMemsetAsync(g.vlabel + v, 0xff, 4, st));
  const csm_update del{'v', 0, 0, v, 0, 0};
  for (csm_ctx* q : all) {
    int rc = 0;
    if (q != ctx) { q->g = g; rc = stream_after(q->st, st, ctx->ev_fork); }
    if (!rc) rc = index_vertex_update(q->index, g, del, q->st, &q->launches);
    if (!rc && q != ctx) rc = stream_after(st, q->st, q->ev_join);
    if (rc) return rc;
  }
  ctx->graph_version++;
  return CSM_OK;
}

static int run_vertex_update(csm_ctx* ctx, const csm_update* ups, const csm_update& h, csm_result* out,
                             const std::vector<csm_result*>& out_q) {
  cudaStream_t st = ctx->st;
  if (h.is_add && h.id1 < ctx->g.n_cap && h.id1 >= ctx->g.n) { ctx->g.n = h.id1 + 1; ctx->graph_version++; }
  if (!h.is_add && h.id1 < ctx->g.n) {
    int rc = run_vertex_delete(ctx, h.id1);
    if (rc) return rc;
  }
  k_vertex_update<<<1, 32, 0, st>>>(ups, 1, ctx->g, ctx->d_info); CKL();
  CK(cudaMemsetAsync(ctx->d_safe, 0xff, 4, st));
  k_finalize<<<1, 32, 0, st>>>(1, ctx->d_info, ctx->d_count, ctx->d_hash, nullptr, nullptr, nullptr, 0, 0, out); CKL();
  int rc = index_vertex_update(ctx->index, ctx->g, h, st, &ctx->launches);
  if (rc) return rc;
  for (size_t k = 0; k < ctx->attached.size(); k++) {
    csm_ctx* a = ctx->attached[k];
    a->g = ctx->g;
    rc = stream_after(a->st, st, ctx->ev_fork);
    if (rc) return rc;
    k_finalize<<<1, 32, 0, a->st>>>(1, ctx->d_info, a->d_count, a->d_hash, nullptr, nullptr, nullptr, 0, 0,
                                    out_q[k]);
    a->launches++;
    CK(cudaGetLastError());
    rc = index_vertex_update(a->index, ctx->g, h, a->st, &a->launches);
    if (rc) return rc;
  }
  for (csm_ctx* a : ctx->attached) {
    rc = stream_after(st, a->st, a->ev_join);
    if (rc) return rc;
  }
  return CSM_OK;
}

// A batch of B edge updates through a CUDA graph of its launch sequence.
// Batch sizes are rounded up to a power of two (at most max_batch) with
// padding records, so that batches of varying size -- as a serving loop
// forms them -- share a few graphs.
static int run_edge_batch_graph(csm_ctx* ctx, const csm_update* ups, uint32_t B_real, csm_result* out,
                                const std::vector<csm_result*>& out_q) {
  cudaStream_t st = ctx->st;
  uint32_t B = 1;
  while (B < B_real) B <<= 1;
  B = std::min<uint32_t>(B, ctx->bmax);
  std::vector<csm_ctx*> all{ctx};
  all.insert(all.end(), ctx->attached.begin(), ctx->attached.end());
  csm_ctx::GraphEntry* ge = nullptr;
  for (auto& e : ctx->graphs)
    if (e.B == B && e.version == ctx->graph_version) { ge = &e; break; }
  if (!ge) {
    // drop graphs of an older version (at most one per power of two is kept)
    for (size_t i = 0; i < ctx->graphs.size();) {
      if (ctx->graphs[i].version != ctx->graph_version || ctx->graphs.size() >= 18) {
        cudaGraphExecDestroy(ctx->graphs[i].exec);
        ctx->graphs.erase(ctx->graphs.begin() + (long)i);
      } else {
        i++;
      }
    }
    std::vector<uint64_t> l0;
    for (csm_ctx* q : all) l0.push_back(q->launches);
    const uint64_t batches0 = ctx->batches;
    std::vector<csm_result*> stage_q;
    for (csm_ctx* a : ctx->attached) stage_q.push_back(a->d_gres);
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
    ctx->capturing = true;
    int rc = run_edge_batch(ctx, ctx->d_gups, B, ctx->d_gres, stage_q);
    ctx->capturing = false;
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (ce != cudaSuccess) return set_err(CSM_ECUDA, "graph capture: %s", cudaGetErrorString(ce));
    cudaGraphExec_t exec = nullptr;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return set_err(CSM_ECUDA, "graph instantiate: %s", cudaGetErrorString(ce));
    csm_ctx::GraphEntry e{B, ctx->graph_version, exec, {}};
    for (size_t k = 0; k < all.size(); k++) {
      e.launches.push_back(all[k]->launches - l0[k]);
      all[k]->launches = l0[k];  // counted when the graph runs
    }
    ctx->batches = batches0;
    for (csm_ctx* a : ctx->attached) a->batches -= 1;
    ctx->graphs.push_back(e);
    ge = &ctx->graphs.back();
  }
  CK(cudaMemcpyAsync(ctx->d_gups, ups, sizeof(csm_update) * (size_t)B_real, cudaMemcpyDeviceToDevice, st));
  if (B > B_real)
    CK(cudaMemcpyAsync(ctx->d_gups + B_real, ctx->d_gpad, sizeof(csm_update) * (size_t)(B - B_real),
                       cudaMemcpyDeviceToDevice, st));
  CK(cudaGraphLaunch(ge->exec, st));
  CK(cudaMemcpyAsync(out, ctx->d_gres, sizeof(csm_result) * (size_t)B_real, cudaMemcpyDeviceToDevice, st));
  for (size_t k = 0; k < ctx->attached.size(); k++)
    CK(cudaMemcpyAsync(out_q[k], ctx->attached[k]->d_gres, sizeof(csm_result) * (size_t)B_real,
                       cudaMemcpyDeviceToDevice, st));
  for (size_t k = 0; k < all.size(); k++) {
    all[k]->launches += ge->launches[k];
    all[k]->batches++;
  }
  ctx->graph_replays++;
  return CSM_OK;
}

// Keeps the edge table's load below one half (live keys plus deleted slots)
// before the updates `h` of a submit run: refills it from the CSR when the
// deleted slots would push it over, in a table twice as large when the live
// keys alone fill a third.  The counts are upper bounds (every insertion
// record counts as a new edge, every deletion as a deleted slot).
static int edge_table_maintain(csm_ctx* ctx, const csm_update* h, uint64_t n) {
  DevGraph& g = ctx->g;
  if (!g.emask) return CSM_OK;
  uint64_t ins = 0, del = 0;
  for (uint64_t i = 0; i < n; i++) {
    if (h[i].type != 'e') continue;
    if (h[i].is_add) ins++; else del++;
  }
  uint64_t slots = g.emask + 1;
  if ((ctx->e_live + ctx->e_tomb + ins + del) * 2 > slots) {
    cudaStream_t st = ctx->st;
    uint64_t want = slots;
    while ((ctx->e_live + ins) * 3 > want) want <<= 1;
    if (want != slots) {
      uint64_t* nk = nullptr;
      CK(cudaStreamSynchronize(st));  // no kernel of an earlier submit still reads the old table
      for (csm_ctx* a : ctx->attached) CK(cudaStreamSynchronize(a->st));
      int rc = ctx->mem.alloc((void**)&nk, 8ull * want);
      if (rc) return rc;
      ctx->mem.release(g.ekeys, 8ull * slots);
      g.ekeys = nk;
      g.emask = want - 1;
      slots = want;
      ctx->graph_version++;  // captured launch sequences hold the old table
    }
    CK(cudaMemsetAsync(g.ekeys, 0xff, 8ull * slots, st));
    k_edge_fill<<<ctx->sm_count * 8, 256, 0, st>>>(g);
    CKL();
    ctx->e_tomb = 0;
  }
  ctx->e_live += ins;
  ctx->e_tomb += del;
  return CSM_OK;
}

static int submit_common(csm_ctx* ctx, uint64_t n, const csm_update* d_ups, const csm_update* h_ups) {
  if (ctx->owner) return set_err(CSM_ESTATE, "updates of an attached query are submitted to its owner");
  if (!ctx->has_graph || !ctx->has_plan) return set_err(CSM_ESTATE, "load the query, the graph and build the index first");
  int rc = ensure_batch_buffers(ctx);
  if (rc) return rc;
  rc = ensure_results(ctx, n);
  if (rc) return rc;
  cudaStream_t st = ctx->st;
  for (csm_ctx* a : ctx->attached) {
    rc = ensure_results(a, n);
    if (!rc) rc = stream_after(st, a->st, a->ev_join);  // work issued on it outside a submit
    if (rc) return rc;
  }
  CK(cudaEventRecord(ctx->ev_start, st));
  if (ctx->d_enum_n) CK(cudaMemsetAsync(ctx->d_enum_n, 0, 16, st));
  for (csm_ctx* a : ctx->attached)
    if (a->d_enum_n) CK(cudaMemsetAsync(a->d_enum_n, 0, 16, st));  // before the fork below
  k_stamp<<<1, 1, 0, st>>>(ctx->d_stamp); CKL();
  for (csm_ctx* a : ctx->attached) {
    rc = stream_after(a->st, st, ctx->ev_fork);
    if (rc) return rc;
    CK(cudaEventRecord(a->ev_start, a->st));
  }
  std::vector<csm_result*> out_q(ctx->attached.size());
  const uint32_t B = (ctx->cfg.mode == CSM_MODE_PLAIN) ? 1u : ctx->bmax;
  // vertex updates run on their own; runs of edge updates form batches
  std::vector<csm_update> hv;
  const csm_update* h = h_ups;
  if (!h) {
    hv.resize(n);
    CK(cudaMemcpyAsync(hv.data(), d_ups, n * sizeof(csm_update), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    h = hv.data();
  }
  rc = edge_table_maintain(ctx, h, n);
  if (rc) return rc;
  uint64_t i = 0;
  while (i < n) {
    for (size_t k = 0; k < ctx->attached.size(); k++) out_q[k] = ctx->attached[k]->d_results + i;
    if (h[i].type == 'v') {
      // the host's mirror of the vertex labels follows the device
      // (k_vertex_update and run_vertex_delete)
      const uint32_t vid = h[i].id1;
      const bool was_added = h[i].is_add && vid < ctx->g.n_cap && ctx->h_vlabel[vid] == kNone;
      const bool removed = !h[i].is_add && vid < ctx->g.n;
      rc = run_vertex_update(ctx, d_ups + i, h[i], ctx->d_results + i, out_q);
      if (rc) return rc;
      if (was_added) ctx->h_vlabel[vid] = fold_host(ctx->qlab_v, h[i].label);
      if (removed) ctx->h_vlabel[vid] = kNone;
      ctx->v_updates++;
      for (csm_ctx* a : ctx->attached) a->v_updates++;
      i++;
      continue;
    }
    if (ctx->cfg.mode == CSM_MODE_PLAIN && ctx->attached.empty() && !ctx->d_enum) {
      rc = run_plain_edge(ctx, d_ups + i, h[i], ctx->d_results + i);
      if (rc) return rc;
      ctx->e_updates++;
      i++;
      continue;
    }
    uint64_t j = i;
    while (j < n && j - i < B && h[j].type != 'v') j++;
    if (ctx->cfg.graphs == CSM_GRAPHS_ON)
      rc = run_edge_batch_graph(ctx, d_ups + i, (uint32_t)(j - i), ctx->d_results + i, out_q);
    else
      rc = run_edge_batch(ctx, d_ups + i, (uint32_t)(j - i), ctx->d_results + i, out_q);
    if (rc) return rc;
    ctx->e_updates += j - i;
    for (csm_ctx* a : ctx->attached) a->e_updates += j - i;
    i = j;
  }
  CK(cudaEventRecord(ctx->ev_end, st));
  std::vector<csm_ctx*> all{ctx};
  all.insert(all.end(), ctx->attached.begin(), ctx->attached.end());
  for (csm_ctx* q : all) {
    if (q != ctx) CK(cudaEventRecord(q->ev_end, q->st));
    q->last_first = q->seq_next;
    q->last_n = n;
    q->seq_next += n;
    q->updates_done += n;
    q->totals_dirty = true;
    q->h_last_valid = false;
  }
  return CSM_OK;
}

// Puts the hand-over ring back into its initial state (after a failed launch).
static int reset_ring(csm_ctx* ctx) {
  if (!ctx->d_q) return CSM_OK;
  CK(cudaMemsetAsync(ctx->d_q, 0, sizeof(SearchQueue), ctx->st));
  std::vector<unsigned long long> seq(ctx->qcap);
  for (uint32_t i = 0; i < ctx->qcap; i++) seq[i] = i;
  CK(cudaMemcpyAsync(ctx->d_qseq, seq.data(), 8ull * ctx->qcap, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return CSM_OK;
}

static int check_device_error(csm_ctx* ctx) {
  PoolState ps;
  CK(cudaMemcpy(&ps, ctx->g.ps, sizeof(PoolState), cudaMemcpyDeviceToHost));
  if (ps.error) {
    static const char* names[] = {"none", "row pool exhausted", "batch list overflow", "task list overflow",
                                  "search queue wait limit", "malformed donated task", "ring left undrained",
                                  "task time guard", "row state", "edge table full"};
    char extra[256] = "";
    if (ctx->d_sstat) {
      SearchStats ss;
      if (cudaMemcpy(&ss, ctx->d_sstat, sizeof(ss), cudaMemcpyDeviceToHost) == cudaSuccess) {
        if (ss.bad_set)
          snprintf(extra, sizeof(extra), " [ticket %llu seq %llu words %u %08x %u %u %u batch %u]", ss.bad_ticket,
                   ss.bad_seq, ss.bad_words[0], ss.bad_words[1], ss.bad_words[2], ss.bad_words[3], ss.bad_words[4],
                   ss.bad_batch);
        if (ss.guard_set) {
          int o = snprintf(extra, sizeof(extra), " [guard d %u upd %u iters %llu lv", ss.guard_d, ss.guard_upd,
                           ss.guard_iters);
          for (unsigned L = 0; L < ss.guard_d && L < 16 && o < (int)sizeof(extra) - 40; L++)
            o += snprintf(extra + o, sizeof(extra) - o, " %u/%u/%u/%u", ss.guard_lv[4 * L], ss.guard_lv[4 * L + 1],
                          ss.guard_lv[4 * L + 2], ss.guard_lv[4 * L + 3]);
          snprintf(extra + o, sizeof(extra) - o, "]");
        }
      }
    }
    const unsigned int code = ps.error;
    ps.error = 0;
    cudaMemcpy(ctx->g.ps, &ps, sizeof(PoolState), cudaMemcpyHostToDevice);
    reset_ring(ctx);
    return set_err(CSM_EDEVICE, "device error %u (%s)%s", code, code < 10 ? names[code] : "?", extra);
  }
  return CSM_OK;
}

// Sums the search-kernel event pairs of completed submits.
static int collect_search_times(csm_ctx* ctx) {
  for (size_t i = 0; i < ctx->sev_used; i++) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->sev[i].first, ctx->sev[i].second));
    ctx->search_ms += ms;
  }
  ctx->search_launches += ctx->sev_used;
  ctx->sev_used = 0;
  return CSM_OK;
}

static int fetch_last(csm_ctx* ctx) {
  if (ctx->h_last_valid) return CSM_OK;
  CK(cudaStreamSynchronize(ctx->st));
  {
    int rc0 = collect_search_times(ctx);
    if (rc0) return rc0;
  }
  int rc = check_device_error(ctx);
  if (rc) return rc;
  ctx->h_last.resize(ctx->last_n);
  if (ctx->last_n) {
    CK(cudaMemcpyAsync(ctx->h_last.data(), ctx->d_results, ctx->last_n * sizeof(csm_result), cudaMemcpyDeviceToHost,
                       ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  if (ctx->totals_dirty) {
    for (const csm_result& r : ctx->h_last) {
      ctx->tot_pos += r.pos; ctx->tot_neg += r.neg;
      if (r.pos || r.neg) ctx->tot_unsafe++;
      ctx->work_bytes += r.work_bytes;
    }
    ctx->totals_dirty = false;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_end) == cudaSuccess) { ctx->last_ms = ms; ctx->total_ms += ms; }
  }
  ctx->h_last_valid = true;
  return CSM_OK;
}

}  // namespace csm

// ================================================================== C ABI

// ------------------------------------------------------------ autotuner
//
// The search's launch shape -- warps per block (each warp walks one subtree
// at a time, so this sets how many subtrees share a block's shared memory)
// and resident blocks per SM -- is chosen per query and graph by timing the
// search on a sample of update edges for every shape the SM admits (shared
// memory of the per-warp level buffers, 32 warps of 64 registers per SM).
// The sample is searched as insertions against the current graph, which is
// not modified: each edge's seeds run the ordinary search with positions 0
// and 1 fixed, whether or not the edge is present.

__global__ void k_tune_prep(const csm_update* edges, uint32_t n, DevGraph g, UpdInfo* info) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const csm_update u = edges[i];
  UpdInfo inf;
  inf.v1 = u.id1; inf.v2 = u.id2; inf.label = fold_elabel(g, u.label);
  const bool ok = u.type == 'e' && u.id1 < g.n && u.id2 < g.n && u.id1 != u.id2 && g.vlabel[u.id1] != kNone &&
                  g.vlabel[u.id2] != kNone;
  inf.flags = ok ? (UF_VALID | UF_ADD) : UF_INVALID;
  info[i] = inf;
}

static int tune_run(csm_ctx* ctx, uint32_t B, uint32_t warps, uint32_t bps, float* ms, uint32_t donate_every = 0,
                    uint32_t split_deep = 0) {
  cudaStream_t st = ctx->st;
  const DevGraph& g = ctx->g;
  unsigned int* c = ctx->d_cnt;
  CK(cudaMemsetAsync(c, 0, 64, st));
  CK(cudaMemsetAsync(ctx->d_count, 0, 8ull * B, st));
  CK(cudaMemsetAsync(ctx->d_bytes, 0, 8ull * B, st));
  CK(cudaMemsetAsync(ctx->d_stop, 0, 4ull * B, st));
  k_seed<<<blocks_for(B, 128), 128, 0, st>>>(B, ctx->d_info, g, ctx->d_plan, ctx->index.d2, ctx->index.words,
                                              ctx->d_tasks, c + 6, ctx->task_cap, ctx->d_safe, &g.ps->error); CKL();
  SearchParams sp{};
  sp.g = g; sp.plan = ctx->d_plan; sp.tasks = ctx->d_tasks; sp.n_tasks = c + 6; sp.task_cap = ctx->task_cap;
  sp.task_next = c + 7; sp.info = ctx->d_info; sp.count = ctx->d_count; sp.hash = ctx->d_hash;
  sp.bytes = ctx->d_bytes; sp.stop = ctx->d_stop;
  sp.d2 = ctx->index.d2; sp.d2_words = ctx->index.words; sp.cap = ctx->cfg.max_results;
  sp.homo = ctx->cfg.homomorphism; sp.want_hash = 0; sp.error = &g.ps->error;
  sp.q = ctx->d_q; sp.dq = ctx->d_dq; sp.qseq = ctx->d_qseq; sp.qcap = ctx->qcap;
  sp.wait_limit_ns = 30ull * 1000000000ull;
  sp.slot_limit_ns = 100ull * 1000000ull;
  sp.task_limit_ns = 20ull * 1000000000ull;
  sp.batch = B;
  sp.sstat = ctx->d_sstat;
  sp.donate_every = donate_every;
  sp.split_deep = split_deep;
  sp.tail = (!ctx->cfg.want_hash && !ctx->d_enum && !ctx->cfg.tail_enumerate) ? 1u : 0u;  // as the batches run
  CK(cudaEventRecord(ctx->ev_start, st));
  launch_search(sp, ctx->nq, (uint32_t)ctx->sm_count * bps, warps, st); CKL();
  CK(cudaEventRecord(ctx->ev_end, st));
  CK(cudaEventSynchronize(ctx->ev_end));
  CK(cudaEventElapsedTime(ms, ctx->ev_start, ctx->ev_end));
  return check_device_error(ctx);
}

static int autotune(csm_ctx* ctx, uint32_t n, const csm_update* h_edges, uint32_t* out_w, uint32_t* out_b,
                    float* out_ms) {
  const uint32_t B = std::min<uint32_t>(n, ctx->bmax);
  int rc = ensure_stream(ctx, B);
  if (rc) return rc;
  CK(cudaMemcpyAsync(ctx->d_stream, h_edges, B * sizeof(csm_update), cudaMemcpyHostToDevice, ctx->st));
  k_tune_prep<<<blocks_for(B, 256), 256, 0, ctx->st>>>(ctx->d_stream, B, ctx->g, ctx->d_info); CKL();
  float ms = 0;
  rc = tune_run(ctx, B, 8, 1, &ms);  // warm-up (caches, clocks)
  if (rc) return rc;
  // the default shape (8 warps, every resident block), then the others; a
  // shape replaces the default only when it is at least 5 % faster, since
  // capped updates make single timings vary by a few percent
  const int kmode = ctx->d_enum ? 1 : ((!ctx->cfg.want_hash && !ctx->cfg.tail_enumerate) ? 2 : 0);  // as the batches run
  uint32_t best_w = 8, best_b = std::max<uint32_t>(1, search_max_blocks(ctx->nq, 8, kmode));
  float best = 0;
  rc = tune_run(ctx, B, best_w, best_b, &best);
  if (rc) return rc;
  const float def_ms = best;
  for (uint32_t w : {4u, 8u, 16u}) {
    const uint32_t bmax = search_max_blocks(ctx->nq, w, kmode);  // resident blocks per SM
    for (uint32_t b = std::max<uint32_t>(1, bmax > 3 ? bmax - 3 : 1); b <= bmax; b++) {
      if (w == 8 && b == std::max<uint32_t>(1, search_max_blocks(ctx->nq, 8, kmode))) continue;
      rc = tune_run(ctx, B, w, b, &ms);
      if (rc) return rc;
      if (ms < best && ms < 0.95f * def_ms) { best = ms; best_w = w; best_b = b; }
    }
  }
  // hand-over settings for the chosen shape, against the default (every step, 64)
  uint32_t best_every = 0, best_split = 0;
  const float shape_ms = best;
  static const uint32_t kHandOver[4][2] = {{2u, 64u}, {4u, 64u}, {1u, 16u}, {1u, 256u}};
  for (const auto& cand : kHandOver) {
    rc = tune_run(ctx, B, best_w, best_b, &ms, cand[0], cand[1]);
    if (rc) return rc;
    if (ms < best && ms < 0.95f * shape_ms) { best = ms; best_every = cand[0]; best_split = cand[1]; }
  }
  ctx->cfg.donate_every = best_every;
  ctx->cfg.split_deep = best_split;
  ctx->cfg.warps_per_block = best_w;
  ctx->cfg.blocks_per_sm = best_b;
  ctx->graph_version++;
  if (ctx->owner) ctx->owner->graph_version++;
  *out_w = best_w; *out_b = best_b; *out_ms = best;
  return CSM_OK;
}

// ------------------------------------------------------------ initial match

// InitialMatching() (ParaCOSM/CSM/matching/GraphFlow/graphflow.cpp:268-284,
// SymBi/symbi.cpp:374-402): the number of embeddings of the query in the
// current graph, without the per-update cap.  Every embedding maps the first
// anchor query edge (u_a, u_b) onto exactly one directed data entry
// (m[u_a], m[u_b]), so the entries of S(x, L(u_b), l(u_a, u_b)) over the
// vertices x of label L(u_a) are the seeds: each becomes a root task of the
// ordinary search (positions 0 and 1 fixed) and the per-seed counts are summed.

__global__ void k_init_count(DevGraph g, uint32_t la, uint32_t combo, unsigned long long* cnt) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= g.n_cap) return;
  unsigned long long c = 0;
  if (v < g.n && g.vlabel[v] == la) {
    const uint32_t* d = g.dir + (size_t)v * (g.nc + 1) + combo;
    c = d[1] - d[0];
  }
  cnt[v] = c;
}

// Seeds [first, first + B) of the entry enumeration: info and one task each.
__global__ void k_init_fill(DevGraph g, uint32_t combo, uint32_t label, const unsigned long long* off,
                            unsigned long long first, uint32_t B, uint32_t stride, uint32_t rank, UpdInfo* info,
                            Task* tasks) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B) return;
  const unsigned long long e = (first + i) * stride + rank;  // this shard's seeds
  uint32_t lo = 0, hi = g.n_cap;  // last x with off[x] <= e
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= e) lo = mid; else hi = mid;
  }
  const uint32_t x = lo;
  const uint32_t* pool = g.pools[g.ps->active];
  const uint32_t* d = g.dir + (size_t)x * (g.nc + 1) + combo;
  const uint32_t y = pool[g.row_off[x] + d[0] + (e - off[x])];
  UpdInfo u;
  u.v1 = x; u.v2 = y; u.label = label; u.flags = UF_VALID | UF_ADD;
  info[i] = u;
  tasks[i] = Task{i, 0, 0, 0};
}

__global__ void k_init_sum(uint32_t B, const unsigned long long* count, unsigned long long* total) {
  unsigned long long s = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x) s += count[i];
#pragma unroll
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(total, s);
}

static int initial_match(csm_ctx* ctx, uint64_t* out) {
  cudaStream_t st = ctx->st;
  DevGraph& g = ctx->g;
  const PlanAnchor& A = ctx->h_plan->anchors[0];
  const uint32_t combo = A.lb * g.n_el + A.el;
  const uint64_t n_cap = g.n_cap;
  unsigned long long *cnt = nullptr, *off = nullptr, *total = nullptr;
  void* tmp = nullptr;
  size_t tb = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, off, (int64_t)n_cap, st));
  int rc = ctx->mem.alloc((void**)&cnt, 8ull * n_cap);
  if (!rc) rc = ctx->mem.alloc((void**)&off, 8ull * n_cap);
  if (!rc) rc = ctx->mem.alloc((void**)&total, 64);
  if (!rc) rc = ctx->mem.alloc(&tmp, tb);
  auto release = [&]() {
    ctx->mem.release(cnt, 8ull * n_cap); ctx->mem.release(off, 8ull * n_cap);
    ctx->mem.release(total, 64); ctx->mem.release(tmp, tb);
  };
  if (rc) { release(); return rc; }
  k_init_count<<<blocks_for(n_cap, 256), 256, 0, st>>>(g, A.la, combo, cnt); CKL();
  CK(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, (int64_t)n_cap, st));
  CK(cudaMemsetAsync(total, 0, 64, st));
  unsigned long long last_off = 0, last_cnt = 0;
  CK(cudaMemcpyAsync(&last_off, off + (n_cap - 1), 8, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&last_cnt, cnt + (n_cap - 1), 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const unsigned long long n_all = last_off + last_cnt;
  // with seed sharding this context takes the seeds e = k * shard_count + shard_rank
  const uint32_t stride = ctx->cfg.shard_count > 1 ? ctx->cfg.shard_count : 1u;
  const uint32_t rank = stride > 1 ? ctx->cfg.shard_rank : 0u;
  const unsigned long long n_seeds = n_all > rank ? (n_all - rank + stride - 1) / stride : 0ull;
  uint32_t warps, bps;
  search_shape(ctx, warps, bps);
  for (unsigned long long first = 0; first < n_seeds; first += ctx->bmax) {
    const uint32_t B = (uint32_t)std::min<unsigned long long>(ctx->bmax, n_seeds - first);
    unsigned int* c = ctx->d_cnt;
    CK(cudaMemsetAsync(c, 0, 64, st));
    CK(cudaMemcpyAsync(c + 6, &B, 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(ctx->d_count, 0, 8ull * B, st));
    CK(cudaMemsetAsync(ctx->d_bytes, 0, 8ull * B, st));
    CK(cudaMemsetAsync(ctx->d_stop, 0, 4ull * B, st));
    k_init_fill<<<blocks_for(B, 256), 256, 0, st>>>(g, combo, A.el, off, first, B, stride, rank, ctx->d_info,
                                                    ctx->d_tasks); CKL();
    SearchParams sp{};
    sp.g = g; sp.plan = ctx->d_plan; sp.tasks = ctx->d_tasks; sp.n_tasks = c + 6; sp.task_cap = ctx->task_cap;
    sp.task_next = c + 7; sp.info = ctx->d_info; sp.count = ctx->d_count; sp.hash = ctx->d_hash;
    sp.bytes = ctx->d_bytes; sp.stop = ctx->d_stop;
    sp.d2 = ctx->index.d2; sp.d2_words = ctx->index.words; sp.cap = 0;
    sp.homo = ctx->cfg.homomorphism; sp.want_hash = 0; sp.error = &g.ps->error;
    sp.q = ctx->d_q; sp.dq = ctx->d_dq; sp.qseq = ctx->d_qseq; sp.qcap = ctx->qcap;
    sp.wait_limit_ns = 30ull * 1000000000ull;
    sp.slot_limit_ns = 100ull * 1000000ull;
    sp.task_limit_ns = 20ull * 1000000000ull;
    sp.batch = B;
    sp.sstat = ctx->d_sstat;
    sp.tail = ctx->cfg.tail_enumerate ? 0u : 1u;
    launch_search(sp, ctx->nq, (uint32_t)ctx->sm_count * bps, warps, st); CKL();
    ctx->search_launches++;
    k_init_sum<<<std::min<uint32_t>(blocks_for(B, 256), 1024), 256, 0, st>>>(B, ctx->d_count, total); CKL();
    ctx->launches += 3;
  }
  unsigned long long h = 0;
  CK(cudaMemcpyAsync(&h, total, 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  release();
  rc = check_device_error(ctx);
  if (rc) return rc;
  *out = h;
  return CSM_OK;
}

extern "C" {

void csm_gpu_default_cfg(csm_cfg* cfg) {
  memset(cfg, 0, sizeof(*cfg));
  cfg->algorithm = CSM_ALGO_GRAPHFLOW;
  cfg->mode = CSM_MODE_BATCHED;
  cfg->max_batch = kMaxBatch;
}

const char* csm_gpu_last_error(void) { return g_last_error.c_str(); }

const char* csm_gpu_strerror(int code) {
  switch (code) {
    case CSM_OK: return "ok";
    case CSM_EINVAL: return "invalid argument";
    case CSM_ENOMEM: return "out of device memory or HBM budget";
    case CSM_ECUDA: return "CUDA error";
    case CSM_ESTATE: return "call out of order";
    case CSM_EUNSUPPORTED: return "unsupported input";
    case CSM_ETIMEOUT: return "timed out";
    case CSM_EDEVICE: return "device-side error";
    default: return "unknown error";
  }
}

int csm_gpu_create(const csm_cfg* cfg, csm_ctx** out) {
  if (!cfg || !out) return set_err(CSM_EINVAL, "null argument");
  if (cfg->algorithm < 0 || cfg->algorithm > CSM_ALGO_NEWSP)
    return set_err(CSM_EINVAL, "unknown algorithm %d", cfg->algorithm);
  if (cfg->max_batch > kMaxBatch) return set_err(CSM_EINVAL, "max_batch above %u", kMaxBatch);
  if (cfg->shard_count > 1 && cfg->shard_rank >= cfg->shard_count)
    return set_err(CSM_EINVAL, "shard_rank %u outside shard_count %u", cfg->shard_rank, cfg->shard_count);
  if (cfg->enum_capacity && cfg->graphs == CSM_GRAPHS_ON)
    return set_err(CSM_EUNSUPPORTED, "match-set output (enum_capacity) cannot be combined with graph replay");
  if (cfg->turboflux_compat && (cfg->algorithm != CSM_ALGO_TURBOFLUX || cfg->mode != CSM_MODE_PLAIN))
    return set_err(CSM_EUNSUPPORTED, "turboflux_compat needs the TurboFlux plugin in CSM_MODE_PLAIN (its deletion "
                                     "count depends on the exact index at each update)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(CSM_ECUDA, "no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev) return set_err(CSM_EINVAL, "bad device %d", cfg->device);
  CK(cudaSetDevice(cfg->device));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, cfg->device));
  if (prop.major < 10) return set_err(CSM_EUNSUPPORTED, "needs an sm_100 device, found sm_%d%d", prop.major, prop.minor);
  csm_ctx* ctx = new csm_ctx();
  ctx->cfg = *cfg;
  if (!ctx->cfg.max_batch) ctx->cfg.max_batch = kMaxBatch;
  ctx->bmax = ctx->cfg.mode == CSM_MODE_PLAIN ? 1u : ctx->cfg.max_batch;
  ctx->dev = cfg->device;
  ctx->sm_count = prop.multiProcessorCount;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  ctx->mem.budget = cfg->hbm_budget_bytes ? cfg->hbm_budget_bytes : (uint64_t)(0.9 * (double)free_b);
  if (cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ctx->ev_start) != cudaSuccess || cudaEventCreate(&ctx->ev_end) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    delete ctx;
    return set_err(CSM_ECUDA, "stream/event creation failed");
  }
  ctx->h_plan = new Plan();
  *out = ctx;
  return CSM_OK;
}

// Query graph of a context: sorted adjacency like Graph::AddEdge (repeats
// ignored), connectivity and size limits.  Label folding is set by the caller.
static int parse_query(csm_ctx* ctx, uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges) {
  if (n_qv < 2 || n_qv > kMaxQ) return set_err(CSM_EUNSUPPORTED, "query must have 2..%u vertices", kMaxQ);
  ctx->nq = n_qv;
  ctx->qvl.assign(q_vlabels, q_vlabels + n_qv);
  for (uint32_t l : ctx->qvl) if (l == kNone) return set_err(CSM_EINVAL, "query vertex without a label");
  ctx->qnbr.assign(n_qv, {});
  ctx->qel.assign(n_qv, {});
  ctx->qe.clear();
  for (uint32_t i = 0; i < n_qe; i++) {
    const uint32_t a = q_edges[3 * i], b = q_edges[3 * i + 1], l = q_edges[3 * i + 2];
    if (a >= n_qv || b >= n_qv) return set_err(CSM_EINVAL, "query edge endpoint out of range");
    if (a == b) continue;
    auto it = std::lower_bound(ctx->qnbr[a].begin(), ctx->qnbr[a].end(), b);
    if (it != ctx->qnbr[a].end() && *it == b) continue;  // Graph::AddEdge: repeat is a no-op
    size_t d = (size_t)(it - ctx->qnbr[a].begin());
    ctx->qnbr[a].insert(it, b); ctx->qel[a].insert(ctx->qel[a].begin() + (long)d, l);
    it = std::lower_bound(ctx->qnbr[b].begin(), ctx->qnbr[b].end(), a);
    d = (size_t)(it - ctx->qnbr[b].begin());
    ctx->qnbr[b].insert(it, a); ctx->qel[b].insert(ctx->qel[b].begin() + (long)d, l);
    ctx->qe.push_back(a); ctx->qe.push_back(b); ctx->qe.push_back(l);
  }
  if (ctx->qe.empty()) return set_err(CSM_EINVAL, "query has no edges");
  {  // the edge-anchored search needs a connected query
    std::vector<char> seen(n_qv, 0);
    std::vector<uint32_t> stack{0};
    seen[0] = 1;
    uint32_t reached = 1;
    while (!stack.empty()) {
      uint32_t u = stack.back(); stack.pop_back();
      for (uint32_t w : ctx->qnbr[u]) if (!seen[w]) { seen[w] = 1; reached++; stack.push_back(w); }
    }
    if (reached != n_qv) return set_err(CSM_EUNSUPPORTED, "query graph is not connected");
  }
  if (ctx->qe.size() / 3 > kMaxQE) return set_err(CSM_EUNSUPPORTED, "query has more than %u edges", kMaxQE);
  return CSM_OK;
}

// Folded query labels from the context's folding tables.
static void fold_query(csm_ctx* ctx) {
  ctx->qvl_f.resize(ctx->nq);
  for (uint32_t u = 0; u < ctx->nq; u++) ctx->qvl_f[u] = fold_host(ctx->qlab_v, ctx->qvl[u]);
}

int csm_gpu_set_query(csm_ctx* ctx, uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe, const uint32_t* q_edges) {
  if (!ctx || !q_vlabels || (n_qe && !q_edges)) return set_err(CSM_EINVAL, "null argument");
  if (ctx->owner) return set_err(CSM_ESTATE, "an attached query is set by csm_gpu_attach_query");
  if (ctx->has_graph) return set_err(CSM_ESTATE, "set the query before loading the graph");
  int rc = parse_query(ctx, n_qv, q_vlabels, n_qe, q_edges);
  if (rc) return rc;
  ctx->qlab_v = ctx->qvl;
  std::sort(ctx->qlab_v.begin(), ctx->qlab_v.end());
  ctx->qlab_v.erase(std::unique(ctx->qlab_v.begin(), ctx->qlab_v.end()), ctx->qlab_v.end());
  ctx->qlab_e.clear();
  for (size_t i = 0; i < ctx->qe.size(); i += 3) ctx->qlab_e.push_back(ctx->qe[i + 2]);
  std::sort(ctx->qlab_e.begin(), ctx->qlab_e.end());
  ctx->qlab_e.erase(std::unique(ctx->qlab_e.begin(), ctx->qlab_e.end()), ctx->qlab_e.end());
  if (ctx->qlab_e.size() + 1 > 64) return set_err(CSM_EUNSUPPORTED, "at most 63 distinct query edge labels");
  fold_query(ctx);
  ctx->has_query = true;
  return CSM_OK;
}

int csm_gpu_reserve_labels(csm_ctx* ctx, uint32_t n_vl, const uint32_t* vlabels, uint32_t n_el, const uint32_t* elabels) {
  if (!ctx || (n_vl && !vlabels) || (n_el && !elabels)) return set_err(CSM_EINVAL, "null argument");
  if (!ctx->has_query || ctx->owner) return set_err(CSM_ESTATE, "set the query of an owning context first");
  if (ctx->has_graph) return set_err(CSM_ESTATE, "reserve labels before loading the graph");
  for (uint32_t i = 0; i < n_vl; i++) {
    if (vlabels[i] == kNone) return set_err(CSM_EINVAL, "label 0xffffffff is reserved for absent vertices");
    ctx->qlab_v.push_back(vlabels[i]);
  }
  for (uint32_t i = 0; i < n_el; i++) ctx->qlab_e.push_back(elabels[i]);
  std::sort(ctx->qlab_v.begin(), ctx->qlab_v.end());
  ctx->qlab_v.erase(std::unique(ctx->qlab_v.begin(), ctx->qlab_v.end()), ctx->qlab_v.end());
  std::sort(ctx->qlab_e.begin(), ctx->qlab_e.end());
  ctx->qlab_e.erase(std::unique(ctx->qlab_e.begin(), ctx->qlab_e.end()), ctx->qlab_e.end());
  if (ctx->qlab_e.size() + 1 > 64) return set_err(CSM_EUNSUPPORTED, "at most 63 distinct edge labels");
  if (ctx->qlab_v.size() + 1 > 4096) return set_err(CSM_EUNSUPPORTED, "at most 4095 distinct vertex labels");
  fold_query(ctx);
  return CSM_OK;
}

int csm_gpu_attach_query(csm_ctx* owner, const csm_cfg* cfg, uint32_t n_qv, const uint32_t* q_vlabels,
                         uint32_t n_qe, const uint32_t* q_edges, csm_ctx** out) {
  if (!owner || !cfg || !out || !q_vlabels || (n_qe && !q_edges)) return set_err(CSM_EINVAL, "null argument");
  if (owner->owner) return set_err(CSM_ESTATE, "attach to the context that owns the graph");
  if (!owner->has_graph || !owner->has_plan) return set_err(CSM_ESTATE, "the owner needs a graph and a built index");
  if (cfg->algorithm < 0 || cfg->algorithm > CSM_ALGO_NEWSP)
    return set_err(CSM_EINVAL, "unknown algorithm %d", cfg->algorithm);
  CK(cudaSetDevice(owner->dev));
  CK(cudaStreamSynchronize(owner->st));
  csm_ctx* a = new csm_ctx();
  a->cfg = owner->cfg;
  a->cfg.algorithm = cfg->algorithm;
  a->cfg.max_results = cfg->max_results;
  a->cfg.tail_enumerate = cfg->tail_enumerate;
  a->cfg.want_hash = cfg->want_hash;
  a->cfg.warps_per_block = cfg->warps_per_block;
  a->cfg.blocks_per_sm = cfg->blocks_per_sm;
  a->cfg.turboflux_compat = cfg->turboflux_compat;
  a->cfg.hbm_budget_bytes = cfg->hbm_budget_bytes;
  a->cfg.enum_capacity = owner->cfg.graphs == CSM_GRAPHS_ON ? 0u : cfg->enum_capacity;
  a->bmax = owner->bmax;
  a->dev = owner->dev;
  a->sm_count = owner->sm_count;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  a->mem.budget = cfg->hbm_budget_bytes ? cfg->hbm_budget_bytes : (uint64_t)(0.9 * (double)free_b);
  auto fail = [&](int rc) { csm_gpu_destroy(a); return rc; };
  if (cudaStreamCreateWithFlags(&a->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&a->ev_start) != cudaSuccess || cudaEventCreate(&a->ev_end) != cudaSuccess ||
      cudaEventCreateWithFlags(&a->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&a->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return fail(set_err(CSM_ECUDA, "stream/event creation failed"));
  a->h_plan = new Plan();
  int rc = parse_query(a, n_qv, q_vlabels, n_qe, q_edges);
  if (rc) return fail(rc);
  // the owner's label folding: every label of this query must be one it keeps
  a->qlab_v = owner->qlab_v;
  a->qlab_e = owner->qlab_e;
  fold_query(a);
  for (uint32_t u = 0; u < a->nq; u++)
    if (a->qvl_f[u] == (uint32_t)a->qlab_v.size())
      return fail(set_err(CSM_EUNSUPPORTED, "vertex label %u is not kept by the owner (csm_gpu_reserve_labels)",
                          a->qvl[u]));
  for (size_t i = 0; i < a->qe.size(); i += 3)
    if (fold_host(a->qlab_e, a->qe[i + 2]) == (uint32_t)a->qlab_e.size())
      return fail(set_err(CSM_EUNSUPPORTED, "edge label %u is not kept by the owner (csm_gpu_reserve_labels)",
                          a->qe[i + 2]));
  a->has_query = true;
  a->g = owner->g;
  a->has_graph = true;
  a->num_edges = owner->num_edges;
  rc = build_plan(a);
  if (!rc) rc = ensure_batch_buffers(a);
  if (!rc) {
    std::vector<std::vector<uint32_t>> qel_f(a->nq);
    for (uint32_t u = 0; u < a->nq; u++)
      for (uint32_t l : a->qel[u]) qel_f[u].push_back(fold_host(a->qlab_e, l));
    IndexQuery q{a->nq, &a->qvl_f, &a->qnbr, &qel_f, a->cfg.homomorphism != 0};
    rc = index_build(a->index, a->mem, a->g, q, a->cfg.algorithm, a->sm_count, a->st, &a->launches);
  }
  if (rc) return fail(rc);
  a->seq_next = owner->seq_next;
  a->owner = owner;
  owner->attached.push_back(a);
  owner->graph_version++;
  *out = a;
  return CSM_OK;
}

int csm_gpu_load_graph(csm_ctx* ctx, uint32_t n_v, const uint32_t* vlabels, uint64_t n_e, const uint32_t* edges) {
  if (!ctx || (n_v && !vlabels) || (n_e && !edges)) return set_err(CSM_EINVAL, "null argument");
  if (!ctx->has_query) return set_err(CSM_ESTATE, "set the query first");
  if (ctx->has_graph) return set_err(CSM_ESTATE, "graph already loaded");
  CK(cudaSetDevice(ctx->dev));
  cudaStream_t st = ctx->st;
  // folded label spaces: the query's distinct labels plus one inert label each
  const uint32_t n_vl = (uint32_t)ctx->qlab_v.size() + 1;
  const uint32_t n_el = (uint32_t)ctx->qlab_e.size() + 1;
  const uint64_t nc = (uint64_t)n_vl * n_el;
  if (nc > 65535) return set_err(CSM_EUNSUPPORTED, "%llu label combinations (at most 65535)", (unsigned long long)nc);
  const uint32_t headroom = ctx->cfg.vertex_headroom ? ctx->cfg.vertex_headroom : 1024;
  const uint64_t n_cap64 = (uint64_t)n_v + headroom;
  if (n_cap64 > (1ull << 30)) return set_err(CSM_EUNSUPPORTED, "too many vertices");
  const uint32_t n_cap = (uint32_t)n_cap64;
  KeyBits kb{ceil_log2((uint64_t)n_cap + 2), std::max<uint32_t>(1, ceil_log2(nc))};
  if (kb.total() > 64) return set_err(CSM_EUNSUPPORTED, "vertex id and label widths exceed a 64-bit key");
  DevGraph& g = ctx->g;
  g.n = n_v; g.n_cap = n_cap; g.n_vl = n_vl; g.n_el = n_el; g.nc = (uint32_t)nc; g.kb = kb;
  DevMem& m = ctx->mem;
  int rc = 0;
#define AL(p, sz) do { rc = m.alloc((void**)&(p), (sz)); if (rc) return rc; } while (0)
  AL(g.vlabel, 4ull * n_cap);
  AL(g.row_off, 8ull * n_cap);
  AL(g.row_cap, 4ull * n_cap);
  AL(g.dir, 4ull * n_cap * (nc + 1));
  AL(g.t_start, 4ull * n_cap);
  AL(g.t_count, 4ull * n_cap);
  AL(g.ps, sizeof(PoolState));
  AL(ctx->d_qlab, 4ull * (ctx->qlab_v.size() + ctx->qlab_e.size()));
  CK(cudaMemcpyAsync(ctx->d_qlab, ctx->qlab_v.data(), 4ull * ctx->qlab_v.size(), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_qlab + ctx->qlab_v.size(), ctx->qlab_e.data(), 4ull * ctx->qlab_e.size(),
                     cudaMemcpyHostToDevice, st));
  g.qlab_v = ctx->d_qlab;
  g.qlab_e = ctx->d_qlab + ctx->qlab_v.size();
  g.n_qv = (uint32_t)ctx->qlab_v.size();
  g.n_qe = (uint32_t)ctx->qlab_e.size();
  CK(cudaMemsetAsync(g.vlabel, 0xff, 4ull * n_cap, st));
  CK(cudaMemcpyAsync(g.vlabel, vlabels, 4ull * n_v, cudaMemcpyHostToDevice, st));
  ctx->h_vlabel.assign(n_cap, kNone);
  for (uint32_t v = 0; v < n_v; v++)
    if (vlabels[v] != kNone) ctx->h_vlabel[v] = fold_host(ctx->qlab_v, vlabels[v]);
  if (n_v) { k_fold_vlabels<<<blocks_for(n_v, 256), 256, 0, st>>>(g.vlabel, n_v, g); CKL(); }
  CK(cudaMemsetAsync(g.row_off, 0, 8ull * n_cap, st));
  CK(cudaMemsetAsync(g.row_cap, 0, 4ull * n_cap, st));
  CK(cudaMemsetAsync(g.dir, 0, 4ull * n_cap * (nc + 1), st));
  CK(cudaMemsetAsync(g.t_count, 0, 4ull * n_cap, st));
  CK(cudaMemsetAsync(g.ps, 0, sizeof(PoolState), st));
  // temporaries
  uint32_t* d_e = nullptr; uint64_t *ukey = nullptr, *ukey2 = nullptr, *uidx = nullptr, *uidx2 = nullptr;
  uint64_t *dkey = nullptr, *dkey2 = nullptr, *first = nullptr, *cap64 = nullptr;
  unsigned long long* d_small = nullptr;
  const uint64_t M = 2 * n_e;
  AL(d_e, 12ull * n_e);
  AL(ukey, 8ull * n_e); AL(ukey2, 8ull * n_e); AL(uidx, 8ull * n_e); AL(uidx2, 8ull * n_e);
  AL(d_small, 64);
  CK(cudaMemcpyAsync(d_e, edges, 12ull * n_e, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(d_small, 0, 64, st));
  if (n_e) { k_load_edge_keys<<<blocks_for(n_e, 256), 256, 0, st>>>(d_e, n_e, g.vlabel, n_v, ukey, uidx, d_small); CKL(); }
  void* tmp = nullptr; size_t tb = 0, tb2 = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, ukey, ukey2, uidx, uidx2, (int64_t)n_e, 0, 64, st));
  CK(cub::DeviceRadixSort::SortKeys(nullptr, tb2, dkey, dkey2, (int64_t)M, 0, (int)kb.total(), st));
  size_t tb3 = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb3, cap64, g.row_off, (int64_t)n_cap, st));
  const size_t tbmax = std::max(tb, std::max(tb2, tb3));
  AL(tmp, tbmax);
  if (n_e) {
    tb = tbmax;
    CK(cub::DeviceRadixSort::SortPairs(tmp, tb, ukey, ukey2, uidx, uidx2, (int64_t)n_e, 0, 64, st));
  }
  unsigned long long bad = 0;
  CK(cudaMemcpyAsync(&bad, d_small, 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  m.release(ukey, 8ull * n_e); m.release(uidx, 8ull * n_e);
  if (bad) { m.release(d_e, 12ull * n_e); m.release(ukey2, 8ull * n_e); m.release(uidx2, 8ull * n_e);
             m.release(tmp, tbmax); m.release(d_small, 64);
             return set_err(CSM_EINVAL, "%llu edges touch a vertex id without a label line", bad); }
  AL(dkey, 8ull * std::max<uint64_t>(M, 1)); AL(dkey2, 8ull * std::max<uint64_t>(M, 1));
  if (n_e) { k_load_directed<<<blocks_for(n_e, 256), 256, 0, st>>>(ukey2, uidx2, n_e, d_e, g, dkey); CKL(); }
  m.release(ukey2, 8ull * n_e); m.release(uidx2, 8ull * n_e); m.release(d_e, 12ull * n_e);
  if (M) {
    tb = tbmax;
    CK(cub::DeviceRadixSort::SortKeys(tmp, tb, dkey, dkey2, (int64_t)M, 0, (int)kb.total(), st));
  }
  m.release(dkey, 8ull * std::max<uint64_t>(M, 1));
  AL(first, 8ull * n_cap); AL(cap64, 8ull * n_cap);
  if (M) { k_load_count<<<blocks_for(M, 256), 256, 0, st>>>(dkey2, M, kb, (uint32_t)nc, g.dir, first, d_small + 1); CKL(); }
  k_dir_scan<<<blocks_for(n_cap, 256), 256, 0, st>>>(g.dir, n_cap, (uint32_t)nc); CKL();
  k_load_caps<<<blocks_for(n_cap, 256), 256, 0, st>>>(g.dir, n_cap, (uint32_t)nc, g.row_cap, cap64); CKL();
  tb = tbmax;
  CK(cub::DeviceScan::ExclusiveSum(tmp, tb, cap64, g.row_off, (int64_t)n_cap, st));
  unsigned long long last_off = 0, last_cap = 0, n_valid = 0;
  CK(cudaMemcpyAsync(&last_off, g.row_off + (n_cap - 1), 8, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&last_cap, cap64 + (n_cap - 1), 8, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&n_valid, d_small + 1, 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const uint64_t used = last_off + last_cap;
  const uint64_t pool_cap = std::max<uint64_t>(2 * used + 16ull * ctx->bmax + (1ull << 20), 1ull << 20);
  if (pool_cap >= (1ull << 32)) return set_err(CSM_EUNSUPPORTED, "graph too large for 32-bit pool offsets");
  g.pool_cap = pool_cap;
  AL(g.pools[0], 4ull * pool_cap);
  AL(g.pools[1], 4ull * pool_cap);
  if (M) { k_load_scatter<<<blocks_for(M, 256), 256, 0, st>>>(dkey2, M, kb, first, g.row_off, g.pools[0]); CKL(); }
  PoolState ps{};
  ps.top[0] = used;
  CK(cudaMemcpyAsync(g.ps, &ps, sizeof(ps), cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  m.release(dkey2, 8ull * std::max<uint64_t>(M, 1)); m.release(first, 8ull * n_cap); m.release(cap64, 8ull * n_cap);
  m.release(tmp, tbmax); m.release(d_small, 64);
#undef AL
  ctx->num_edges = n_valid / 2;
  // edge table: four slots per edge (a power of two); without room for it,
  // or for ids of 30 bits and more or over 16 folded edge labels, the
  // search joins by binary search in the rows instead
  g.ekeys = nullptr;
  g.emask = 0;
  if (n_cap < (1u << 30) && n_el <= 16) {
    uint64_t slots = 1ull << 20;
    while (slots < 4 * std::max<uint64_t>(ctx->num_edges, 1)) slots <<= 1;
    uint64_t* ek = nullptr;
    if (m.alloc((void**)&ek, 8ull * slots) == CSM_OK) {
      g.ekeys = ek;
      g.emask = slots - 1;
      CK(cudaMemsetAsync(g.ekeys, 0xff, 8ull * slots, st));
      k_edge_fill<<<ctx->sm_count * 8, 256, 0, st>>>(g);
      CK(cudaGetLastError());
      CK(cudaStreamSynchronize(st));
      ctx->e_live = ctx->num_edges;
      ctx->e_tomb = 0;
    } else {
      set_err(CSM_OK, "");  // the table is optional
    }
  }
  ctx->has_graph = true;
  return CSM_OK;
}

int csm_gpu_build_index(csm_ctx* ctx) {
  if (!ctx) return set_err(CSM_EINVAL, "null context");
  if (!ctx->has_graph) return set_err(CSM_ESTATE, "load the graph first");
  CK(cudaSetDevice(ctx->dev));
  int rc = build_plan(ctx);
  if (rc) return rc;
  rc = ensure_batch_buffers(ctx);
  if (rc) return rc;
  std::vector<std::vector<uint32_t>> qel_f(ctx->nq);
  for (uint32_t u = 0; u < ctx->nq; u++)
    for (uint32_t l : ctx->qel[u]) qel_f[u].push_back(fold_host(ctx->qlab_e, l));
  IndexQuery q{ctx->nq, &ctx->qvl_f, &ctx->qnbr, &qel_f, ctx->cfg.homomorphism != 0};
  rc = index_build(ctx->index, ctx->mem, ctx->g, q, ctx->cfg.algorithm, ctx->sm_count, ctx->st, &ctx->launches);
  if (rc || !ctx->cfg.turboflux_compat) return rc;
  // compat deletions need to know which anchors are spanning-tree edges
  const IxDag& D = ctx->index.h_dag;
  for (uint32_t a = 0; a < ctx->h_plan->n_anchor; a++) {
    PlanAnchor& A = ctx->h_plan->anchors[a];
    const uint32_t x = A.pos[0].qv, y = A.pos[1].qv;
    bool tree = false;
    for (uint32_t k = 0; k < D.npar[y]; k++) tree |= D.par[y][k] == x;
    for (uint32_t k = 0; k < D.npar[x]; k++) tree |= D.par[x][k] == y;
    A.tree = tree ? 1u : 0u;
  }
  CK(cudaMemcpyAsync(ctx->d_plan, ctx->h_plan, ctx->plan_bytes, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return CSM_OK;
}

int csm_gpu_initial_match(csm_ctx* ctx, uint64_t* count) {
  if (!ctx || !count) return set_err(CSM_EINVAL, "null argument");
  if (!ctx->has_graph || !ctx->has_plan) return set_err(CSM_ESTATE, "load the query, the graph and build the index first");
  CK(cudaSetDevice(ctx->dev));
  int rc = ensure_batch_buffers(ctx);
  if (rc) return rc;
  if (ctx->owner) {  // an attached query reads the owner's graph after the owner's queued work
    ctx->g = ctx->owner->g;
    rc = stream_after(ctx->st, ctx->owner->st, ctx->ev_fork);
    if (rc) return rc;
  }
  return initial_match(ctx, count);
}

int csm_gpu_autotune(csm_ctx* ctx, uint32_t n, const csm_update* edges, uint32_t* warps_per_block,
                     uint32_t* blocks_per_sm, uint32_t* donate_every, uint32_t* split_deep, float* search_ms) {
  if (!ctx || !edges || !warps_per_block || !blocks_per_sm || !donate_every || !split_deep || !search_ms)
    return set_err(CSM_EINVAL, "null argument");
  if (!ctx->has_graph || !ctx->has_plan) return set_err(CSM_ESTATE, "load the query, the graph and build the index first");
  if (n == 0) return set_err(CSM_EINVAL, "empty sample");
  CK(cudaSetDevice(ctx->dev));
  int rc = ensure_batch_buffers(ctx);
  if (rc) return rc;
  if (ctx->owner) {
    ctx->g = ctx->owner->g;
    rc = stream_after(ctx->st, ctx->owner->st, ctx->ev_fork);
    if (rc) return rc;
  }
  rc = autotune(ctx, n, edges, warps_per_block, blocks_per_sm, search_ms);
  *donate_every = ctx->cfg.donate_every;
  *split_deep = ctx->cfg.split_deep;
  return rc;
}

int csm_gpu_classify(csm_ctx* ctx, uint64_t n, const csm_update* ups, uint8_t* safe_out) {
  if (!ctx || (n && (!ups || !safe_out))) return set_err(CSM_EINVAL, "null argument");
  if (!ctx->has_plan) return set_err(CSM_ESTATE, "build the index first");
  if (!n) return CSM_OK;
  int rc = ensure_stream(ctx, n);
  if (rc) return rc;
  uint8_t* d_safe = nullptr;
  rc = ctx->mem.alloc((void**)&d_safe, n);
  if (rc) return rc;
  CK(cudaMemcpyAsync(ctx->d_stream, ups, n * sizeof(csm_update), cudaMemcpyHostToDevice, ctx->st));
  k_classify<<<blocks_for(n, 256), 256, 0, ctx->st>>>(n, ctx->d_stream, ctx->g, ctx->d_plan, d_safe); CKL();
  CK(cudaMemcpyAsync(safe_out, d_safe, n, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->mem.release(d_safe, n);
  return CSM_OK;
}

int csm_gpu_submit(csm_ctx* ctx, uint64_t n, const csm_update* ups) {
  if (!ctx || (n && !ups)) return set_err(CSM_EINVAL, "null argument");
  CK(cudaSetDevice(ctx->dev));
  if (!n) return CSM_OK;
  int rc = ensure_stream(ctx, n);
  if (rc) return rc;
  CK(cudaMemcpyAsync(ctx->d_stream, ups, n * sizeof(csm_update), cudaMemcpyHostToDevice, ctx->st));
  return submit_common(ctx, n, ctx->d_stream, ups);
}

int csm_gpu_submit_device(csm_ctx* ctx, uint64_t n, const csm_update* d_ups) {
  if (!ctx || (n && !d_ups)) return set_err(CSM_EINVAL, "null argument");
  CK(cudaSetDevice(ctx->dev));
  if (!n) return CSM_OK;
  return submit_common(ctx, n, d_ups, nullptr);
}

int csm_gpu_poll(csm_ctx* ctx, int* done) {
  if (!ctx || !done) return set_err(CSM_EINVAL, "null argument");
  CK(cudaSetDevice(ctx->dev));
  cudaError_t e = cudaEventQuery(ctx->ev_end);
  if (e == cudaSuccess && ctx->owner) e = cudaEventQuery(ctx->owner->ev_end);  // the owner issues its work
  if (e == cudaErrorNotReady) { *done = 0; return CSM_OK; }
  if (e != cudaSuccess) return set_err(CSM_ECUDA, "poll: %s", cudaGetErrorString(e));
  *done = 1;
  return CSM_OK;
}

int csm_gpu_wait(csm_ctx* ctx, uint64_t timeout_ns) {
  if (!ctx) return set_err(CSM_EINVAL, "null context");
  if (timeout_ns) {
    auto t0 = std::chrono::steady_clock::now();
    while (cudaEventQuery(ctx->ev_end) == cudaErrorNotReady) {
      if ((uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count() > timeout_ns)
        return set_err(CSM_ETIMEOUT, "wait timed out");
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
  CK(cudaStreamSynchronize(ctx->st));
  int rc = collect_search_times(ctx);
  if (rc) return rc;
  return check_device_error(ctx);
}

int csm_gpu_results(csm_ctx* ctx, uint64_t first_seq, uint64_t n, csm_result* out) {
  if (!ctx || (n && !out)) return set_err(CSM_EINVAL, "null argument");
  if (first_seq < ctx->last_first || first_seq + n > ctx->last_first + ctx->last_n)
    return set_err(CSM_EINVAL, "results are kept for the last submit only: [%llu, %llu)",
                   (unsigned long long)ctx->last_first, (unsigned long long)(ctx->last_first + ctx->last_n));
  int rc = fetch_last(ctx);
  if (rc) return rc;
  memcpy(out, ctx->h_last.data() + (first_seq - ctx->last_first), n * sizeof(csm_result));
  return CSM_OK;
}

int csm_gpu_results_device(csm_ctx* ctx, const csm_result** d_out, uint64_t* n) {
  if (!ctx || !d_out || !n) return set_err(CSM_EINVAL, "null argument");
  *d_out = ctx->d_results;
  *n = ctx->last_n;
  return CSM_OK;
}

int csm_gpu_stats(csm_ctx* ctx, csm_stats* out) {
  if (!ctx || !out) return set_err(CSM_EINVAL, "null argument");
  int rc = fetch_last(ctx);
  if (rc) return rc;
  memset(out, 0, sizeof(*out));
  out->num_vertices = ctx->g.n;
  out->updates_done = ctx->updates_done;
  out->vertex_updates = ctx->v_updates;
  out->edge_updates = ctx->e_updates;
  out->positive = ctx->tot_pos; out->negative = ctx->tot_neg; out->unsafe_updates = ctx->tot_unsafe;
  out->batches = ctx->batches;
  out->kernel_launches = ctx->launches;
  out->device_bytes = ctx->mem.bytes;
  out->pool_capacity = ctx->g.pool_cap;
  out->last_batch_ms = ctx->last_ms;
  out->total_device_ms = ctx->total_ms;
  if (ctx->has_graph) {
    PoolState ps;
    CK(cudaMemcpy(&ps, ctx->g.ps, sizeof(ps), cudaMemcpyDeviceToHost));
    out->pool_entries = ps.top[ps.active];
  }
  {
    uint64_t d1c = 0, d2c = 0;
    int irc = index_counts(ctx->index, ctx->st, &d1c, &d2c);
    if (irc) return irc;
  }
  index_stats(ctx->index, &out->index_entries, &out->index_vertices);
  out->num_edges = ctx->num_edges;
  if (ctx->d_q) {
    SearchQueue q;
    CK(cudaMemcpy(&q, ctx->d_q, sizeof(q), cudaMemcpyDeviceToHost));
    out->donated_tasks = q.tail;
    SearchStats ss;
    CK(cudaMemcpy(&ss, ctx->d_sstat, sizeof(ss), cudaMemcpyDeviceToHost));
    out->search_busy_ns = ss.busy_ns; out->search_idle_ns = ss.idle_ns; out->search_iters = ss.iters;
    out->search_donations = ss.donations; out->search_starved = ss.starved;
  }
  out->search_launches = ctx->search_launches;
  out->search_ms = ctx->search_ms;
  out->work_bytes = ctx->work_bytes;
  return CSM_OK;
}

uint64_t csm_gpu_kernel_launches(csm_ctx* ctx) { return ctx ? ctx->launches : 0; }

void* csm_gpu_stream(csm_ctx* ctx) { return ctx ? (void*)ctx->st : nullptr; }

int csm_gpu_index_info(csm_ctx* ctx, csm_index_info* out) {
  if (!ctx || !out) return set_err(CSM_EINVAL, "null argument");
  CK(cudaSetDevice(ctx->dev));
  memset(out, 0, sizeof(*out));
  out->algorithm = ctx->cfg.algorithm;
  const IndexState& ix = ctx->index;
  if (!ix.active) { out->algorithm = CSM_ALGO_GRAPHFLOW; return CSM_OK; }
  out->n_qv = ix.h_dag.nq;
  out->root = ix.root;
  out->words = ix.words;
  for (uint32_t i = 0; i < ix.h_dag.nq; i++) {
    out->order[i] = ix.order[i];
    uint32_t m = 0;
    for (uint32_t k = 0; k < ix.h_dag.npar[i]; k++) m |= 1u << ix.h_dag.par[i][k];
    out->parents[i] = m;
  }
  return index_counts(ctx->index, ctx->st, &out->d1_count, &out->d2_count);
}

int csm_gpu_index_flags(csm_ctx* ctx, uint32_t which, uint64_t* out, uint64_t out_words) {
  if (!ctx || !out) return set_err(CSM_EINVAL, "null argument");
  const IndexState& ix = ctx->index;
  if (!ix.active) return set_err(CSM_ESTATE, "no candidate index (GraphFlow, or build_index not called)");
  if (which != 1 && which != 2) return set_err(CSM_EINVAL, "which must be 1 (d1) or 2 (d2)");
  if (out_words < ix.words) return set_err(CSM_EINVAL, "out_words below %llu", (unsigned long long)ix.words);
  CK(cudaSetDevice(ctx->dev));
  const uint64_t* src = which == 1 ? ix.bits.d1 : ix.bits.d2;
  CK(cudaMemcpy2DAsync(out, 8ull * out_words, src, 8ull * ix.words, 8ull * ix.words, ix.h_dag.nq,
                       cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (out_words > ix.words)
    for (uint32_t u = 0; u < ix.h_dag.nq; u++)
      memset(out + (uint64_t)u * out_words + ix.words, 0, 8ull * (out_words - ix.words));
  return CSM_OK;
}

int csm_gpu_matches(csm_ctx* ctx, uint32_t* out, uint64_t max_records, uint64_t* n_records, uint64_t* n_found) {
  if (!ctx || !n_records || !n_found || (max_records && !out)) return set_err(CSM_EINVAL, "null argument");
  if (!ctx->d_enum) return set_err(CSM_ESTATE, "match-set output is off (cfg.enum_capacity = 0)");
  CK(cudaSetDevice(ctx->dev));
  int rc = fetch_last(ctx);
  if (rc) return rc;
  unsigned long long found = 0;
  CK(cudaMemcpy(&found, ctx->d_enum_n, 8, cudaMemcpyDeviceToHost));
  const uint64_t kept = std::min<uint64_t>(found, ctx->cfg.enum_capacity);
  const uint64_t n = std::min<uint64_t>(kept, max_records);
  if (n) CK(cudaMemcpy(out, ctx->d_enum, 4ull * (1 + ctx->nq) * n, cudaMemcpyDeviceToHost));
  *n_records = n;
  *n_found = found;
  return CSM_OK;
}

int csm_gpu_search_counters(csm_ctx* ctx, uint64_t* out, uint32_t n) {
  if (!ctx || (n && !out)) return set_err(CSM_EINVAL, "null argument");
  if (!ctx->d_sstat) { for (uint32_t i = 0; i < n; i++) out[i] = 0; return CSM_OK; }
  CK(cudaStreamSynchronize(ctx->st));
  SearchStats ss;
  CK(cudaMemcpy(&ss, ctx->d_sstat, sizeof(ss), cudaMemcpyDeviceToHost));
  const uint64_t v[10] = {ss.busy_ns, ss.idle_ns, ss.iters, ss.donations, ss.starved, ss.checks, ss.checks_hungry,
                          ss.root_busy_ns, ss.last_root_ns, ss.max_task_ns};
  for (uint32_t i = 0; i < n && i < 10; i++) out[i] = v[i];
  return CSM_OK;
}

void csm_gpu_destroy(csm_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->dev);
  cudaStreamSynchronize(ctx->st);
  if (ctx->owner) {  // an attached query leaves its owner's list
    auto& v = ctx->owner->attached;
    v.erase(std::remove(v.begin(), v.end(), ctx), v.end());
    ctx->owner->graph_version++;
  }
  for (auto& e : ctx->graphs) cudaGraphExecDestroy(e.exec);
  ctx->graphs.clear();
  for (csm_ctx* a : ctx->attached) {  // attached queries lose their graph; their calls then fail
    cudaStreamSynchronize(a->st);
    a->owner = nullptr;
    a->has_graph = false;
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  index_free(ctx->index, ctx->mem);
  ctx->mem.free_all();
  for (auto& e : ctx->sev) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_end) cudaEventDestroy(ctx->ev_end);
  if (ctx->st) cudaStreamDestroy(ctx->st);
  delete ctx->h_plan;
  delete ctx;
}

}  // extern "C"

namespace csm {

// Read-only device view of a context, for entry points defined in other
// translation units.
struct CtxView {
  DevGraph g;
  const Plan* plan;
  const uint64_t* d2;
  uint64_t d2_words;
  uint32_t nq, n_anchor;
  int sm_count, device;
  cudaStream_t st;
  uint64_t cap;
  int homo, want_hash;
  uint32_t warps, bps;
  uint32_t dup_zero;       // CaLiG: an insertion of a present edge counts 0
  cudaEvent_t owner_end;   // attached query: end of the owner's last submit (null otherwise)
};

bool ctx_view(csm_ctx* ctx, CtxView* v) {
  if (!ctx || !v || !ctx->has_graph || !ctx->has_plan) return false;
  if (ctx->owner && !ctx->owner->has_graph) return false;
  // an attached query reads its owner's graph, which the owner's submits
  // mutate on the owner's stream
  v->g = ctx->owner ? ctx->owner->g : ctx->g;
  v->owner_end = ctx->owner ? ctx->owner->ev_end : nullptr;
  v->dup_zero = ctx->cfg.algorithm == CSM_ALGO_CALIG ? 1u : 0u;
  v->plan = ctx->d_plan;
  v->d2 = ctx->index.d2;
  v->d2_words = ctx->index.words;
  v->nq = ctx->nq;
  v->n_anchor = ctx->h_plan->n_anchor;
  v->sm_count = ctx->sm_count;
  v->device = ctx->dev;
  v->st = ctx->st;
  v->cap = ctx->cfg.max_results;
  v->homo = ctx->cfg.homomorphism;
  v->want_hash = ctx->cfg.want_hash;
  // the launch shape of the submit path's enumerating search (the probe does
  // not count tails)
  uint32_t warps = ctx->cfg.warps_per_block ? ctx->cfg.warps_per_block : 8;
  if (warps != 4 && warps != 8 && warps != 16) warps = 8;
  uint32_t bps = ctx->cfg.blocks_per_sm;
  if (!bps) bps = std::max<uint32_t>(1, search_max_blocks(ctx->nq, warps, 0));
  v->warps = warps;
  v->bps = bps;
  return true;
}

}  // namespace csm
