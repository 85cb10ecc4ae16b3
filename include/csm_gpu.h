/*
 * csm_gpu.h - C ABI of the B200 continuous-subgraph-matching engine.
 *
 * The engine replaces the hot path behind the reference's plugin interface
 * `class matching` (ParaCOSM/CSM/matching/matching.h:9-66) for the plugins
 * `parallel_graphflow`, `parallel_turboflux` and `parallel_symbi`
 * (ParaCOSM/CSM/matching/main.cpp:740-757), and the reference's standalone
 * CaLiG program (ParaCOSM/CSM/matching/Parallel_CaLiG/parallel_calig.cpp).  A C++ host (paracosm_b200/host)
 * wraps these entry points in `matching`-style plugin classes so that the
 * csm command line and its output lines are unchanged.
 *
 * Labels are arbitrary uint32 values.  Internally every vertex label and
 * edge label that the query does not use is folded into one "inert" label:
 * such vertices and edges can never be part of an embedding, but they stay
 * in the graph, so duplicate inserts and deletions behave as in the
 * reference.
 *
 * Conventions
 *   - Every int-returning call returns CSM_OK (0) or a negative CSM_E* code;
 *     nothing calls exit() (the reference exits on bad input,
 *     ParaCOSM/CSM/graph/graph.cpp:98-109).  csm_gpu_last_error() gives text.
 *   - Input buffers are host memory owned by the caller for the duration of
 *     the call only; the library copies what it keeps.  The *_device variants
 *     take device pointers instead.
 *   - One context is used by one host thread at a time.
 *   - All ids and labels are uint32; counts are uint64.
 *   - Results keep the sequential update order's semantics
 *     (ParaCOSM/CSM/matching/main.cpp:628-674): an insertion counts the
 *     embeddings containing the new edge after adding it, a deletion counts
 *     them before removing it, and every update sees the graph left by all
 *     earlier updates, whether updates are run one per launch or batched.
 */
#ifndef CSM_GPU_H
#define CSM_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ---------------------------------------------------- */
#define CSM_OK 0
#define CSM_EINVAL -1       /* bad argument */
#define CSM_ENOMEM -2       /* device memory or HBM budget exhausted */
#define CSM_ECUDA -3        /* CUDA runtime error */
#define CSM_ESTATE -4       /* call out of order (e.g. submit before load) */
#define CSM_EUNSUPPORTED -5 /* input outside the supported limits */
#define CSM_ETIMEOUT -6     /* csm_gpu_wait deadline passed */
#define CSM_EDEVICE -7      /* a kernel reported an internal error flag */

/* ---- per-update status (csm_result.status) -------------------------- */
#define CSM_ST_OK 0         /* exact count */
#define CSM_ST_CAPPED 1     /* count reached max_results; reported count == max_results */
#define CSM_ST_TIMED_OUT 2  /* per-update deadline reached; count is a lower bound */
#define CSM_ST_INVALID 3    /* e.g. deleting a missing edge; count 0, graph unchanged */

/* ---- algorithms (the reference's -a names) -------------------------- */
#define CSM_ALGO_GRAPHFLOW 0 /* -a parallel_graphflow / graphflow: no index */
#define CSM_ALGO_TURBOFLUX 1 /* -a parallel_turboflux / turboflux: DCG over a query spanning tree */
#define CSM_ALGO_SYMBI 2     /* -a parallel_symbi / symbi: DCS over a DAG of all query edges */
#define CSM_ALGO_CALIG 3     /* -a parallel_calig / calig: CaLiG-style lighting filter over every query edge;
                                an insertion of a present edge counts 0 (Parallel_CaLiG/parallel_calig.cpp:1249) */
#define CSM_ALGO_NEWSP 4     /* -a parallel_newsp / newsp: NewSP-style neighbour-label-frequency filter
                                (Parallel_NewSP/matching/CSMPP.cpp:81-113 indexCheck); leaf vertices counted
                                together when only counts are wanted (its isolated vertices, :641) */

/* ---- execution modes ------------------------------------------------ */
#define CSM_MODE_BATCHED 0   /* many updates per launch sequence (default) */
#define CSM_MODE_PLAIN 1     /* one update per launch sequence: 2-3 launches for an update whose label
                                triple matches no query edge, about 9 otherwise (index marks and one
                                cooperative index round, seeds, search, results) */

typedef struct csm_cfg {
  int32_t algorithm;          /* CSM_ALGO_* */
  int32_t homomorphism;       /* != 0: drop the injectivity check (reference --homo) */
  uint64_t max_results;       /* per-update cap (reference --max-results); 0 = none */
  uint64_t deadline_ns;       /* per-update time budget, counted on the device from the start of the
                                 search launch that holds the update; past it the update stops and
                                 reports CSM_ST_TIMED_OUT with its count so far; 0 = none */
  uint64_t hbm_budget_bytes;  /* device memory the context may hold; 0 = 90% of free */
  int32_t mode;               /* CSM_MODE_* */
  uint32_t max_batch;         /* updates per batch in CSM_MODE_BATCHED (<= 65536); 0 = 65536 */
  int32_t want_hash;          /* != 0: compute the per-update match-set hash */
  int32_t device;             /* CUDA device ordinal */
  int32_t turboflux_compat;   /* != 0: reproduce the reference TurboFlux deletion count, which
                                 seeds every query edge whose vertex labels match, ignoring the
                                 anchor's edge label, and filters anchor endpoints by d2 only on
                                 spanning-tree edges (ParaCOSM/CSM/matching/TurboFlux/
                                 turboflux.cpp:966-1022); TurboFlux in CSM_MODE_PLAIN only */
  uint32_t warps_per_block;   /* search kernel tuning; 0 = autotuned */
  uint32_t blocks_per_sm;     /* search kernel tuning; 0 = autotuned */
  uint32_t vertex_headroom;   /* vertex slots beyond the loaded graph for 'v' updates; 0 = 1024 */
  int32_t graphs;             /* CSM_GRAPHS_*: replay each batch's launch sequence as a CUDA graph */
  uint32_t shard_rank;        /* seed sharding across GPUs: this context searches only the root tasks */
  uint32_t shard_count;       /* (update, anchor, orientation) with (update + 2 * anchor + orientation)
                                 % shard_count == shard_rank; the per-update results of all shards sum
                                 to the unsharded ones (counts capped at max_results after the sum).
                                 shard_count 0 or 1: no sharding */
  uint32_t donate_every;      /* search hand-over check interval in steps (power of two); 0 = autotuned / 1 */
  uint32_t split_deep;        /* smallest driver range split deep in the search tree; 0 = autotuned / 64 */
  uint32_t enum_capacity;     /* > 0: keep up to this many embeddings of each submit (--print-enum,
                                 read with csm_gpu_matches); not with CSM_GRAPHS_ON */
  uint32_t tail_enumerate;    /* when only counts are wanted (want_hash 0, no match sets) the search
                                 counts the last positions of an order that share no query edge as a
                                 product of candidate counts (not in the reference); != 0 enumerates
                                 them one by one instead.  Counts are the same (a product saturates at
                                 2^58 per partial match, beyond any count an enumeration reaches);
                                 work_bytes differ */
} csm_cfg;

#define CSM_GRAPHS_OFF 0      /* launch every kernel of a batch from the host */
#define CSM_GRAPHS_ON 1       /* capture a batch's launch sequence once per batch size and replay it
                                 (search times are then not split out in csm_stats.search_ms); in
                                 CSM_MODE_PLAIN only with attached queries or match-set output, the
                                 other plain updates run their short sequences directly */

/* Same 16-byte layout as the reference's InsertUnit fields
 * (ParaCOSM/CSM/utils/types.h:34-42). */
typedef struct csm_update {
  uint8_t type;     /* 'v' or 'e' */
  uint8_t is_add;   /* 1 = insertion, 0 = deletion */
  uint16_t pad;
  uint32_t id1, id2, label;
} csm_update;

typedef struct csm_result {
  uint64_t pos;     /* positive matches of this update (insertions) */
  uint64_t neg;     /* negative matches of this update (deletions) */
  uint64_t hash;    /* order-independent match-set hash (0 unless want_hash and status OK) */
  uint64_t work_bytes; /* algorithmic bytes: 4 B x the sizes of all back-neighbour segments of
                          every expanded search-tree node, + 16 B per applied edge mutation */
  uint64_t latency_ns; /* submit -> result ready, measured on the device clock */
  uint32_t status;  /* CSM_ST_* */
  uint32_t safe;    /* 1 when the label-triple test (Classify) found no matching query edge */
} csm_result;

typedef struct csm_stats {
  uint64_t num_vertices, num_edges;
  uint64_t updates_done, vertex_updates, edge_updates;
  uint64_t positive, negative, unsafe_updates; /* reference summary counters */
  uint64_t batches, kernel_launches;
  uint64_t search_tasks, donated_tasks;
  uint64_t device_bytes;      /* device memory held by the context */
  uint64_t pool_entries, pool_capacity;
  double last_batch_ms, total_device_ms;
  uint64_t index_entries, index_vertices; /* set d1 / set d2 flags over all query vertices (TurboFlux / SymBi) */
  uint64_t search_launches;   /* launches of the search kernel */
  double search_ms;           /* their summed duration, from CUDA events on the launching stream */
  uint64_t work_bytes;        /* algorithmic bytes of all completed updates (csm_result.work_bytes) */
  uint64_t search_busy_ns;    /* summed warp time inside search tasks */
  uint64_t search_idle_ns;    /* summed warp time waiting for handed-over tasks */
  uint64_t search_iters;      /* chunk iterations (32 candidate slots each) */
  uint64_t search_donations;  /* hand-overs of work between warps */
  uint64_t search_starved;    /* idle warps were waiting but a busy warp had nothing to hand over */
} csm_stats;

typedef struct csm_ctx csm_ctx;

/* Fills *cfg with the defaults. */
void csm_gpu_default_cfg(csm_cfg* cfg);

/* Creates a context on cfg->device (Parallel_* constructors, main.cpp:740-757). */
int csm_gpu_create(const csm_cfg* cfg, csm_ctx** out);

/* Sets the query graph: n_qv vertices with labels, n_qe undirected edges as
 * (u, v, label) triples (Graph::LoadFromFile of -q, graph.cpp:217-249).
 * Must come before csm_gpu_build_index. */
int csm_gpu_set_query(csm_ctx* ctx, uint32_t n_qv, const uint32_t* q_vlabels, uint32_t n_qe,
                      const uint32_t* q_edges);

/* Loads the initial data graph (-d): n_v vertex slots with labels
 * (0xffffffff = absent) and n_e undirected edges as (v1, v2, label) triples.
 * Self loops and repeated edges are dropped (the first label wins). */
int csm_gpu_load_graph(csm_ctx* ctx, uint32_t n_v, const uint32_t* vlabels, uint64_t n_e,
                       const uint32_t* edges);

/* Standing queries sharing one data graph.  The context that loads the graph
 * (the owner) folds labels its query does not use into one inert label; to
 * attach other queries later, first keep their labels distinct with
 * csm_gpu_reserve_labels (between csm_gpu_set_query and csm_gpu_load_graph).
 * The reference runs one query per process (main.cpp:676-871); these two
 * entry points have no reference counterpart. */
int csm_gpu_reserve_labels(csm_ctx* ctx, uint32_t n_vl, const uint32_t* vlabels, uint32_t n_el,
                           const uint32_t* elabels);

/* Attaches a standing query to the owner's graph (after the owner's
 * csm_gpu_build_index), with its own plugin (cfg->algorithm), cap
 * (cfg->max_results), hash and launch-shape settings; device, mode, batch
 * size and homomorphism are the owner's.  The new context has its own plan,
 * candidate index, search buffers and stream.  Updates are submitted to the
 * owner only: every owner submit applies each mutation once and runs every
 * attached query on the same batches, their searches overlapping on the
 * device; each attached context then answers csm_gpu_wait / results / stats /
 * index calls for its query, with the owner's sequence numbers.  Destroying
 * an attached context detaches it; destroying the owner leaves attached
 * contexts without a graph (their calls fail until they are destroyed). */
int csm_gpu_attach_query(csm_ctx* owner, const csm_cfg* cfg, uint32_t n_qv, const uint32_t* q_vlabels,
                         uint32_t n_qe, const uint32_t* q_edges, csm_ctx** out);

/* Preprocessing(): matching orders and, for TurboFlux / SymBi, the auxiliary
 * index (BuildDAG + BuildDCS). */
int csm_gpu_build_index(csm_ctx* ctx);

/* InitialMatching(): number of embeddings in the current graph. */
int csm_gpu_initial_match(csm_ctx* ctx, uint64_t* count);

/* Autotuner: times the search on n sample edges (host memory, type 'e'
 * records; searched as insertions into the current graph, which is not
 * modified) for every launch shape the SM admits -- warps per block x
 * resident blocks per SM -- then for a few hand-over settings (check
 * interval, smallest split range), and keeps the fastest for this context's
 * later searches (a setting replaces the default only when it is at least 5 %
 * faster).  Reports the choice (0 = the default hand-over setting) and its
 * search time on the sample.  The
 * reference tunes its CPU thread count instead (--auto-tuning,
 * ParaCOSM/CSM/matching/Parallel_TurboFlux/parallel_turboflux.cpp); there is
 * no counterpart entry point. */
int csm_gpu_autotune(csm_ctx* ctx, uint32_t n, const csm_update* edges, uint32_t* warps_per_block,
                     uint32_t* blocks_per_sm, uint32_t* donate_every, uint32_t* split_deep, float* search_ms);

/* Classify(v1, v2, label) for n updates: safe_out[i] = 1 when no query edge
 * matches the label triple (L(v1), L(v2), label) in either orientation
 * (ParaCOSM/CSM/matching/Parallel_GraphFlow/parallel_graphflow.cpp:1990-2016). */
int csm_gpu_classify(csm_ctx* ctx, uint64_t n, const csm_update* ups, uint8_t* safe_out);

/* Queues n updates (host memory) after all earlier ones; sequence numbers
 * continue from the previous submit.  Runs asynchronously. */
int csm_gpu_submit(csm_ctx* ctx, uint64_t n, const csm_update* ups);
/* Same, with the updates already in device memory.  Only edge updates are
 * taken from device memory; a vertex update there is reported
 * CSM_ST_INVALID (submit vertex updates from host memory). */
int csm_gpu_submit_device(csm_ctx* ctx, uint64_t n, const csm_update* d_ups);

/* Counts, for each of n edges (v1, v2, label) given in device memory (n <=
 * 1024; csm_update records with type 'e'), the embeddings of the query that
 * contain the edge in the context's current graph -- the count an insertion
 * of an edge already in the graph reports -- into d_counts[i] (device
 * memory, capped at max_results; 0 for an edge with an unknown endpoint).
 * For the CaLiG-style plugin that count is 0: its rule for an insertion of
 * a present edge.  An edge that is not in the graph is searched as the
 * anchor all the same, against the current candidate index (exact for
 * GraphFlow; for the index plugins the insertion itself may add candidates
 * that this count misses).  The probe counts the whole graph (a seed-sharded
 * context's shard settings and the per-update deadline do not apply), and on
 * an attached query it reads the owner's graph after the owner's last
 * submit.  The graph is not modified.  This entry point has no counterpart in the
 * reference.  It is for callers that cannot allocate device memory where
 * they need counts (a locked or stream-ordered memory pool, a latency-
 * critical loop in which an allocation would synchronise the device): it
 * calls no cudaMalloc, cudaFree or allocating library routine, and keeps its
 * working memory in one static device array of 8 MiB per GPU, held while the
 * library is loaded.  The first call on a device resolves that array and
 * initialises it, and should come before any stream capture.  Calls share
 * the array, so calls whose work overlaps on the GPU race.  Runs on the
 * context's stream and waits for it. */
int csm_gpu_probe_noalloc(csm_ctx* ctx, uint32_t n, const csm_update* d_edges, uint64_t* d_counts);

/* Candidate index of the TurboFlux / SymBi plugins: the DAG the index is
 * defined over.  The reference keeps these as private plugin members
 * (q_root_, serialized_tree_, treeNode_[u].backwards_,
 * ParaCOSM/CSM/matching/SymBi/symbi.h:33-44); there is no reference entry
 * point.  They back the index parity tests and debugging. */
typedef struct csm_index_info {
  int32_t algorithm;     /* CSM_ALGO_*; GRAPHFLOW (no index): the rest is zero */
  uint32_t n_qv;
  uint32_t root;         /* q_root_ */
  uint32_t reserved;
  uint64_t words;        /* 64-bit words per flag row */
  uint32_t order[32];    /* serialized_tree_ (a topological order of the DAG) */
  uint32_t parents[32];  /* bitmask of DAG parents per query vertex (treeNode_[u].backwards_) */
  uint64_t d1_count, d2_count;  /* set flags over all query vertices */
} csm_index_info;
int csm_gpu_index_info(csm_ctx* ctx, csm_index_info* out);

/* Copies the d1 (which = 1) or d2 (which = 2) flags (symbi.h:55-56: per
 * query vertex, the data vertices that pass the top-down / the full filter)
 * to host memory as [n_qv][out_words] little-endian bitsets over data vertex
 * ids; out_words must be at least csm_index_info.words.  Waits for the
 * context's stream.  No reference entry point (private members there). */
int csm_gpu_index_flags(csm_ctx* ctx, uint32_t which, uint64_t* out, uint64_t out_words);

/* Embeddings found by the last submit (the reference's --print-enum output,
 * ParaCOSM/CSM/matching/SymBi/symbi.cpp:564-569), when cfg.enum_capacity > 0.
 * Each record is 1 + n_qv uint32 words: the update's index within the last
 * submit, then the data vertex of each query vertex in query-vertex order.
 * Copies min(found, enum_capacity, max_records) records to out; *n_found is
 * every embedding found (more than the capacity means records were dropped).
 * Order is unspecified; with max_results, an update that reaches the cap may
 * list more embeddings than its reported count.  Waits for the stream. */
int csm_gpu_matches(csm_ctx* ctx, uint32_t* out, uint64_t max_records, uint64_t* n_records, uint64_t* n_found);

/* The CUDA stream (cudaStream_t) every launch of this context is issued on,
 * so callers can time work with events on the launching stream. */
void* csm_gpu_stream(csm_ctx* ctx);

/* *done = 1 when every submitted update has a result (the submit's work on
 * the device has finished), else 0; does not block. */
int csm_gpu_poll(csm_ctx* ctx, int* done);

/* Waits until every submitted update has a result, or timeout_ns passes
 * (0 = no limit). */
int csm_gpu_wait(csm_ctx* ctx, uint64_t timeout_ns);

/* Copies results of updates [first_seq, first_seq + n) to host memory.
 * Implies csm_gpu_wait for those updates. */
int csm_gpu_results(csm_ctx* ctx, uint64_t first_seq, uint64_t n, csm_result* out);

/* Device pointer of the result array of the last completed submit (n
 * entries, in submit order); valid until the next submit. */
int csm_gpu_results_device(csm_ctx* ctx, const csm_result** d_out, uint64_t* n);

int csm_gpu_stats(csm_ctx* ctx, csm_stats* out);

/* Search tracing counters, cumulative over the context's search launches:
 * out[0] busy ns, [1] idle ns, [2] chunk iterations, [3] hand-overs,
 * [4] starved checks, [5] hand-over checks, [6] checks that saw idle warps,
 * [7] ns in root tasks, [8] latest root-task end after its launch start (max),
 * [9] longest task ns (max).  Writes min(n, 10) values; waits for the stream. */
int csm_gpu_search_counters(csm_ctx* ctx, uint64_t* out, uint32_t n);

/* Number of distinct kernel launches issued by this context so far. */
uint64_t csm_gpu_kernel_launches(csm_ctx* ctx);

void csm_gpu_destroy(csm_ctx* ctx);

/* Text of the last error on this thread. */
const char* csm_gpu_last_error(void);
const char* csm_gpu_strerror(int code);

#ifdef __cplusplus
}
#endif
#endif /* CSM_GPU_H */
