// csm_gpu_probe_noalloc: edge-embedding counts that allocate no device memory.
//
// Some callers cannot call cudaMalloc on the path where they need counts: a
// host that set the engine up earlier but must not allocate afterwards (a
// locked or stream-ordered memory pool, a latency-critical loop where an
// allocation would synchronise the device, or code that runs while other
// components own the allocator).  This entry point serves them: it reads the
// graph and query an existing context already holds, and keeps all of its
// working memory (task list, hand-over ring, counters) in one file-scope
// static device array, so a call only issues kernels and small copies.
//
// The array is kProbeScratchBytes per GPU and lives as long as the library
// is loaded.  Every call on a device shares it and it keeps the last call's
// contents, so each call clears what must start at zero; calls whose work
// overlaps on the GPU race with each other.  Its layout is fixed (the task
// region is sized for the largest query the engine accepts), so contexts with
// different queries can use it one after another.
#include <cstring>
#include <mutex>

#include "csm_host.cuh"
#include "csm_kernels.cuh"

namespace csm {

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
bool ctx_view(csm_ctx* ctx, CtxView* v);  // csm_api.cu

constexpr uint32_t kProbeMax = 1024;   // edges per call
constexpr uint32_t kProbeRing = 16384; // hand-over ring slots (a power of two, above any grid's warp count)
constexpr size_t kProbeScratchBytes = (size_t)8 << 20;
constexpr int kProbeDevices = 64;

static constexpr size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

// Fixed byte offsets inside the scratch array.
constexpr size_t kOffWords = 0;                                               // [0] tasks [1] next [2] error
constexpr size_t kOffQueue = up256(kOffWords + 64);
constexpr size_t kOffStats = up256(kOffQueue + sizeof(SearchQueue));
constexpr size_t kOffSeq = up256(kOffStats + sizeof(SearchStats));
constexpr size_t kOffRing = up256(kOffSeq + 8ull * kProbeRing);
constexpr size_t kOffInfo = up256(kOffRing + sizeof(DTask) * (size_t)kProbeRing);
constexpr size_t kOffCount = up256(kOffInfo + sizeof(UpdInfo) * kProbeMax);
constexpr size_t kOffHash = up256(kOffCount + 8ull * kProbeMax);
constexpr size_t kOffBytes = up256(kOffHash + 8ull * kProbeMax);
constexpr size_t kOffStop = up256(kOffBytes + 8ull * kProbeMax);
constexpr size_t kOffSafe = up256(kOffStop + 4ull * kProbeMax);
constexpr size_t kOffTasks = up256(kOffSafe + 4ull * kProbeMax);
constexpr size_t kOffEnd = up256(kOffTasks + sizeof(Task) * (size_t)kProbeMax * 2 * kMaxQE);
static_assert(kOffEnd <= kProbeScratchBytes, "probe scratch layout exceeds the array");

// The scratch.  Host code must not use this name as an address: the device
// address is resolved per device with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_probe_scratch[kProbeScratchBytes];

// Ring sequence numbers start at the slot index; the queue starts empty.
__global__ void k_probe_init(unsigned long long* seq, SearchQueue* q) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kProbeRing; i += gridDim.x * blockDim.x) seq[i] = i;
  if (blockIdx.x == 0 && threadIdx.x == 0) { q->head = 0; q->tail = 0; q->hungry = 0; q->pending = 0; }
}

// Per call: the counters that must start at zero, and one UpdInfo per edge.
__global__ void k_probe_prep(const csm_update* edges, uint32_t n, DevGraph g, UpdInfo* info,
                             unsigned long long* count, unsigned long long* hash, unsigned long long* bytes,
                             unsigned int* stop, unsigned int* words, SearchStats* sstat) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    words[0] = 0; words[1] = 0; words[2] = 0;
    memset(sstat, 0, sizeof(SearchStats));
  }
  if (i >= n) return;
  const csm_update u = edges[i];
  UpdInfo inf;
  inf.v1 = u.id1; inf.v2 = u.id2; inf.label = fold_elabel(g, u.label);
  const bool ok = u.type == 'e' && u.id1 < g.n && u.id2 < g.n && u.id1 != u.id2 && g.vlabel[u.id1] != kNone &&
                  g.vlabel[u.id2] != kNone;
  inf.flags = ok ? (UF_VALID | UF_ADD) : UF_INVALID;
  // an edge already in the graph is a duplicate insertion (what the submit
  // path's k_resolve marks): the CaLiG rule counts it 0
  if (ok && find_label(g, g.pools[g.ps->active], u.id1, u.id2) != kNone) inf.flags |= UF_DUP;
  info[i] = inf;
  count[i] = 0; hash[i] = 0; bytes[i] = 0; stop[i] = 0;
}

__global__ void k_probe_out(uint32_t n, const UpdInfo* info, const unsigned long long* count, uint64_t cap,
                            uint64_t* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long c = (info[i].flags & UF_INVALID) ? 0ull : count[i];
  if (cap && c > cap) c = cap;
  out[i] = c;
}

struct ProbeDevice {
  unsigned char* base = nullptr;  // device address of g_probe_scratch on this device
  bool ready = false;
};
static ProbeDevice g_probe_dev[kProbeDevices];
static std::mutex g_probe_mu;

}  // namespace csm

using namespace csm;

extern "C" int csm_gpu_probe_noalloc(csm_ctx* ctx, uint32_t n, const csm_update* d_edges, uint64_t* d_counts) {
  CtxView v;
  if (!ctx_view(ctx, &v)) return set_err(CSM_ESTATE, "probe needs a context with a graph and a built index");
  if (n == 0) return CSM_OK;
  if (!d_edges || !d_counts) return set_err(CSM_EINVAL, "null argument");
  if (n > kProbeMax) return set_err(CSM_EINVAL, "probe takes at most %u edges per call (got %u)", kProbeMax, n);
  if (v.device < 0 || v.device >= kProbeDevices) return set_err(CSM_EUNSUPPORTED, "device ordinal out of range");
  const uint32_t warps_total = (uint32_t)v.sm_count * v.bps * v.warps;
  if (warps_total >= kProbeRing) return set_err(CSM_EUNSUPPORTED, "search grid larger than the probe ring");
  cudaError_t e = cudaSetDevice(v.device);
  if (e != cudaSuccess) return set_err(CSM_ECUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  ProbeDevice& pd = g_probe_dev[v.device];
  {
    // Once per device, with that device current: resolve the array's device
    // address and initialise the ring.  This first call should come before
    // any stream capture.
    std::lock_guard<std::mutex> lk(g_probe_mu);
    if (!pd.ready) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_probe_scratch);
      if (e != cudaSuccess) return set_err(CSM_ECUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      pd.base = static_cast<unsigned char*>(ptr);
      k_probe_init<<<16, 256, 0, v.st>>>(reinterpret_cast<unsigned long long*>(pd.base + kOffSeq),
                                         reinterpret_cast<SearchQueue*>(pd.base + kOffQueue));
      e = cudaStreamSynchronize(v.st);
      if (e != cudaSuccess) return set_err(CSM_ECUDA, "probe set-up: %s", cudaGetErrorString(e));
      pd.ready = true;
    }
  }
  unsigned char* b = pd.base;
  unsigned int* words = reinterpret_cast<unsigned int*>(b + kOffWords);
  SearchQueue* q = reinterpret_cast<SearchQueue*>(b + kOffQueue);
  SearchStats* sstat = reinterpret_cast<SearchStats*>(b + kOffStats);
  unsigned long long* seq = reinterpret_cast<unsigned long long*>(b + kOffSeq);
  DTask* ring = reinterpret_cast<DTask*>(b + kOffRing);
  UpdInfo* info = reinterpret_cast<UpdInfo*>(b + kOffInfo);
  unsigned long long* count = reinterpret_cast<unsigned long long*>(b + kOffCount);
  unsigned long long* hash = reinterpret_cast<unsigned long long*>(b + kOffHash);
  unsigned long long* bytes = reinterpret_cast<unsigned long long*>(b + kOffBytes);
  unsigned int* stop = reinterpret_cast<unsigned int*>(b + kOffStop);
  uint32_t* safe = reinterpret_cast<uint32_t*>(b + kOffSafe);
  Task* tasks = reinterpret_cast<Task*>(b + kOffTasks);

  const uint32_t task_cap = n * 2 * v.n_anchor;
  const uint32_t nb = (n + 255) / 256;
  if (v.owner_end) {
    // an attached query's graph is mutated by its owner's submits, on the
    // owner's stream: read it after the owner's last submit
    e = cudaStreamWaitEvent(v.st, v.owner_end, 0);
    if (e != cudaSuccess) return set_err(CSM_ECUDA, "probe: wait for the owner: %s", cudaGetErrorString(e));
  }
  k_probe_prep<<<nb, 256, 0, v.st>>>(d_edges, n, v.g, info, count, hash, bytes, stop, words, sstat);
  k_seed<<<(n + 127) / 128, 128, 0, v.st>>>(n, info, v.g, v.plan, v.d2, v.d2_words, tasks, words + 0, task_cap, safe,
                                             words + 2, 0, 1, 0, v.dup_zero);
  SearchParams sp{};
  sp.g = v.g; sp.plan = v.plan; sp.tasks = tasks; sp.n_tasks = words + 0; sp.task_cap = task_cap;
  sp.task_next = words + 1; sp.info = info; sp.count = count; sp.hash = hash; sp.bytes = bytes; sp.stop = stop;
  sp.d2 = v.d2; sp.d2_words = v.d2_words; sp.cap = v.cap; sp.homo = v.homo; sp.want_hash = v.want_hash;
  sp.error = words + 2;
  sp.q = q; sp.dq = ring; sp.qseq = seq; sp.qcap = kProbeRing;
  sp.wait_limit_ns = 30ull * 1000000000ull;
  sp.slot_limit_ns = 100ull * 1000000ull;
  sp.task_limit_ns = 20ull * 1000000000ull;
  sp.batch = n;
  sp.sstat = sstat;
  launch_search(sp, v.nq, (uint32_t)v.sm_count * v.bps, v.warps, v.st);
  k_probe_out<<<nb, 256, 0, v.st>>>(n, info, count, v.cap, d_counts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CSM_ECUDA, "probe launch: %s", cudaGetErrorString(e));
  e = cudaStreamSynchronize(v.st);
  if (e != cudaSuccess) return set_err(CSM_ECUDA, "probe: %s", cudaGetErrorString(e));
  unsigned int err = 0;
  e = cudaMemcpyAsync(&err, words + 2, sizeof(err), cudaMemcpyDeviceToHost, v.st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(v.st);
  if (e != cudaSuccess) return set_err(CSM_ECUDA, "probe status: %s", cudaGetErrorString(e));
  if (err) {
    // a failed launch may leave the ring undrained: start it afresh
    k_probe_init<<<16, 256, 0, v.st>>>(seq, q);
    cudaStreamSynchronize(v.st);
    return set_err(CSM_EDEVICE, "probe: device error %u", err);
  }
  return CSM_OK;
}
