// Kernel entry points of the engine (defined in csm_kernels.cu and
// csm_search.cu), launched by the context in csm_api.cu.
#pragma once
#include "csm_internal.cuh"

namespace csm {

// A run of consecutive entries of one vertex in a sorted packed-key list.
struct VRange {
  uint32_t x, start, count, pad;
};

// ---- load-time CSR build (csm_kernels.cu) ----
__global__ void k_load_edge_keys(const uint32_t* e, uint64_t m, const uint32_t* vlabel, uint32_t n,
                                 uint64_t* key, uint64_t* idx, unsigned long long* bad);
__global__ void k_fold_vlabels(uint32_t* vlabel, uint32_t n, DevGraph g);
__global__ void k_load_directed(const uint64_t* ukey, const uint64_t* uidx, uint64_t m, const uint32_t* e,
                                DevGraph g, uint64_t* dkey);
__global__ void k_load_count(const uint64_t* dkey, uint64_t M, KeyBits kb, uint32_t nc, uint32_t* dir,
                             uint64_t* first, unsigned long long* n_valid);
__global__ void k_load_caps(const uint32_t* dir, uint32_t n_cap, uint32_t nc, uint32_t* cap, uint64_t* cap64);
__global__ void k_load_scatter(const uint64_t* dkey, uint64_t M, KeyBits kb, const uint64_t* first,
                               const uint64_t* row_off, uint32_t* pool);
__global__ void k_dir_scan(uint32_t* dir, uint32_t n_cap, uint32_t nc);

// ---- batch preparation ----
__global__ void k_batch_init(const csm_update* ups, uint32_t B, DevGraph g, uint64_t* ukey, uint32_t* useq,
                             UpdInfo* info);
struct ResolveOut {
  uint64_t* ins_key; unsigned int* n_ins;
  uint64_t* del_key; unsigned int* n_del;
  uint64_t* t_key; uint64_t* t_span; unsigned int* n_t;
  uint32_t cap;  // capacity of each list
};
__global__ void k_resolve(const uint64_t* skey, const uint32_t* sseq, uint32_t B, DevGraph g,
                          const csm_update* ups, UpdInfo* info, ResolveOut out);
constexpr uint32_t kBigRow = 4096;  // rows longer than this are mutated by a whole block
__global__ void k_ranges(const uint64_t* key, uint32_t cap, KeyBits kb, VRange* ranges, unsigned int* n_ranges,
                         const uint32_t* dir, uint32_t nc);
__global__ void k_temporal_set(const VRange* ranges, const unsigned int* n_ranges, DevGraph g);
__global__ void k_temporal_clear(const VRange* ranges, const unsigned int* n_ranges, DevGraph g);
__global__ void k_reloc_need(const VRange* ranges, const unsigned int* n_ranges, DevGraph g);
__global__ void k_compact_check(DevGraph g);
__global__ void k_compact_copy(DevGraph g);
__global__ void k_compact_finish(DevGraph g);
void launch_mut_insert(const VRange* ranges, const unsigned int* n_ranges, const uint64_t* ins_key,
                       uint32_t* ins_dst, const DevGraph& g, uint32_t warp_blocks, uint32_t big_blocks,
                       cudaStream_t st);
void launch_mut_delete(const VRange* ranges, const unsigned int* n_ranges, const uint64_t* del_key,
                       uint32_t* del_pos, const DevGraph& g, uint32_t warp_blocks, uint32_t big_blocks,
                       cudaStream_t st);
__global__ void k_vdel_keys(DevGraph g, uint32_t v, uint32_t deg, uint64_t* keys);

// ---- edge table (csm_kernels.cu) ----
// Inserts every (edge, label) of the CSR (one warp per row, from the row of
// the smaller endpoint).
__global__ void k_edge_fill(DevGraph g);
// Inserts (del = 0) or deletes (del = 1) the edges of a packed-key list of
// directed entries (x, combo, y) (the batch lists; each edge appears in both
// directions and is taken from x < y).
__global__ void k_edge_list(const uint64_t* keys, uint32_t L, DevGraph g, uint32_t del);

// ---- one edge update per launch sequence (the plain form; csm_kernels.cu) ----
// keys[0..1]: the update's two directed entries (sentinels when the graph does
// not change); cnt[0..15], count/hash/bytes/stop[0]: cleared for the search.
__global__ void k_plain_resolve(const csm_update* up, DevGraph g, UpdInfo* info, uint64_t* keys, unsigned int* cnt,
                                unsigned long long* count, unsigned long long* hash, unsigned long long* bytes,
                                unsigned int* stop);
// Applies the update's row insertion or deletion (one 256-thread block), after
// finishing a compaction k_compact_copy ran; with `out`, also writes the
// result of an update that needs no search (latency from stamp[0]).
__global__ void k_plain_mutate(DevGraph g, const UpdInfo* info, const uint64_t* keys, csm_result* out,
                               const unsigned long long* stamp, uint32_t mut_bytes);
__global__ void k_vertex_update(const csm_update* ups, uint32_t B, DevGraph g, UpdInfo* info);

// ---- search (csm_search.cu) ----
// Donated search task: a partial match of positions 0..depth (depth 1 = the
// updated edge itself) and the driver range of position depth + 1.
struct DTask {
  uint32_t upd;
  uint16_t anchor;
  uint8_t orient;
  uint8_t depth;
  uint32_t dlo, dn, dsel;
  uint32_t m[kMaxQ];
  uint32_t pad[3];
};
static_assert(sizeof(DTask) == 160, "DTask is 160 bytes");

// Work queue of the search launches.  Tickets count up across launches: an
// idle warp takes ticket `head` (fetch-and-add) and waits for its record; a
// busy warp hands work over by filling tickets from `tail`, one per unit of
// `hungry` it takes (a signed count of idle warps not yet promised a record),
// so records go to waiting warps in ticket order and tail never passes head.
// `pending` counts this launch's tasks (root and donated) that are not
// finished, and waiting warps exit when it reaches zero.
struct SearchQueue {
  unsigned long long head, tail;
  unsigned int hungry, pending;
};

// Cumulative search counters (device memory, read by csm_gpu_stats).
struct SearchStats {
  unsigned long long busy_ns;    // warp time spent inside tasks
  unsigned long long idle_ns;    // warp time spent waiting for handed-over tasks
  unsigned long long iters;      // chunk iterations (32 candidate slots each)
  unsigned long long donations;  // hand-overs (one or more tasks each)
  unsigned long long starved;    // idle warps existed but nothing could be handed over
  unsigned long long checks;     // hand-over checks made by busy warps
  unsigned long long checks_hungry;  // ... that saw idle warps waiting
  unsigned long long root_busy_ns;   // warp time in root tasks (the rest is handed-over tasks)
  unsigned long long last_root_ns;   // max over warps: kernel start -> end of its last root task
  unsigned long long max_task_ns;    // longest single task
  unsigned long long launch_t0;      // globaltimer at the start of the current launch
  // first malformed handed-over record seen: ticket, observed sequence, words 0..4, batch
  unsigned long long bad_ticket, bad_seq;
  unsigned int bad_words[5], bad_batch;
  unsigned int bad_set, pad_;
  // first task stopped by the task time guard: its depth, iterations, update and level cursors
  unsigned int guard_set, guard_d, guard_upd, guard_pad;
  unsigned long long guard_iters;
  unsigned int guard_lv[4 * 16];  // per level 1..16: cnt, cur_e, cur_k, dn[cur_e]
};

struct SearchParams {
  DevGraph g;
  const Plan* plan;
  const Task* tasks;
  const unsigned int* n_tasks;
  uint32_t task_cap;
  unsigned int* task_next;
  const UpdInfo* info;
  unsigned long long* count;   // per update of the batch
  unsigned long long* hash;    // per update of the batch
  unsigned long long* bytes;   // per update: algorithmic bytes of the expanded nodes
  unsigned int* stop;          // per update: cap reached
  const uint64_t* d2;          // optional candidate filter bitsets [n_q][d2_words]
  uint64_t d2_words;
  uint64_t cap;                // 0 = none
  int homo;
  int want_hash;
  unsigned int* error;
  // work donation (null dq: off)
  SearchQueue* q;
  DTask* dq;                  // ring of qcap slots (a power of two)
  unsigned long long* qseq;   // per-slot sequence numbers
  uint32_t qcap;
  unsigned long long wait_limit_ns;  // idle warps waiting for work
  unsigned long long slot_limit_ns;  // a hand-over waiting for its ring slot
  unsigned long long task_limit_ns;  // one task (a guard: a correct walk always ends)
  uint32_t batch;             // updates in this batch (bound of task update indices)
  SearchStats* sstat;
  unsigned long long deadline_ns;  // per-update time budget from the launch's start; 0 = none
  // hand-over tuning: busy warps look for idle ones every donate_every
  // iterations (a power of two; 0 = every iteration) and split a driver range deep in the
  // tree only when at least split_deep elements remain (0 = 64)
  uint32_t donate_every, split_deep;
  // match-set output (null: off): each embedding found at a leaf is appended
  // as a record of 1 + n_q words (enum_base + its update's batch index, then
  // the data vertex of every query vertex in query-vertex order) while fewer
  // than enum_cap records exist; enum_n counts every embedding found
  uint32_t* enum_buf;
  unsigned long long* enum_n;
  unsigned long long enum_cap;
  uint32_t enum_base, enum_stride;
  // nonzero: count each anchor's independent tail (PlanAnchor::tail_at)
  // instead of enumerating it; only for counts without hashes or match sets
  uint32_t tail;
};
__global__ void k_seed(uint32_t B, const UpdInfo* info, DevGraph g, const Plan* plan, const uint64_t* d2,
                       uint64_t d2_words, Task* tasks, unsigned int* n_tasks, uint32_t task_cap,
                       uint32_t* safe, unsigned int* error, uint32_t shard_rank = 0, uint32_t shard_count = 1,
                       uint32_t turboflux_compat = 0, uint32_t dup_zero = 0);
size_t search_smem_bytes(uint32_t n_q, uint32_t warps);
uint32_t search_max_blocks(uint32_t n_q, uint32_t warps, int mode = 0);  // mode: 0 plain, 1 match sets, 2 tail counting
void launch_search(const SearchParams& p, uint32_t n_q, uint32_t blocks, uint32_t warps, cudaStream_t s);
__global__ void k_finalize(uint32_t B, const UpdInfo* info, const unsigned long long* count,
                           const unsigned long long* hash, const unsigned long long* bytes, const uint32_t* safe,
                           const unsigned int* stop, uint64_t cap, int want_hash, csm_result* out,
                           uint32_t mut_bytes = 16,  // bytes of an applied mutation (0 on secondary shards)
                           const unsigned long long* stamp = nullptr);  // non-null: latency from stamp[0]
// stop[] values: 1 = the cap was reached, 2 = the deadline passed first
constexpr unsigned int kStopCap = 1u, kStopDeadline = 2u;
__global__ void k_classify(uint64_t n, const csm_update* ups, DevGraph g, const Plan* plan, uint8_t* safe);

}  // namespace csm
