// Sequential-semantics driver for the reference ParaCOSM plugins.
//
// Built a second time with -DCSM_GPU_PLUGIN (oracle/_ref/ref_driver_gpu), it
// also accepts -a gpu_graphflow / gpu_turboflux / gpu_symbi / gpu_calig /
// gpu_newsp: the CUDA engine as a `matching` subclass (include/
// csm_gpu_plugin.h), driven by this same loop through the reference's
// plugin interface.
//
// Test infrastructure only: this program links the UNMODIFIED reference plugin
// objects (compiled from the reference sources by oracle/ref_build/Makefile)
// and drives them the way the reference's dead `SingleThreadUpdate` loop does
// (ParaCOSM/CSM/matching/main.cpp:628-674): every update is applied in stream
// order and the per-update change of the positive / negative counters is
// recorded.  The shipped `main` instead calls `BatchUpdates3`
// (ParaCOSM/CSM/matching/main.cpp:253-397,822), which skips "safe" updates and
// never applies deletions, so it cannot serve as a per-update oracle.
//
// Plugins are constructed exactly as main.cpp:740-757 does.  With --hash, the
// plugin is created with print_enum=true and every enumeration line it writes
// to std::cout (ParaCOSM/CSM/matching/SymBi/symbi.cpp:564-569,
// ParaCOSM/CSM/matching/TurboFlux/turboflux.cpp:793-798) is parsed and folded
// into an order-independent per-update match-set hash.
//
// Inputs are the reference's text formats (Graph::LoadFromFile /
// LoadUpdateStream, ParaCOSM/CSM/graph/graph.cpp:217-285) or the binary
// container written by the workload generator (loaded by calling
// Graph::AddVertex / Graph::AddEdge in sorted order, which yields the same
// Graph state as the text loader on the same edges).
#include <omp.h>
#include <signal.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <streambuf>
#include <string>
#include <thread>
#include <vector>

#include "graph/graph.h"
#include "matching/GraphFlow/graphflow.h"
#include "matching/Parallel_GraphFlow/parallel_graphflow.h"
#include "matching/Parallel_SymBi/parallel.h"
#include "matching/Parallel_TurboFlux/parallel_turboflux.h"
#include "matching/SymBi/symbi.h"
#include "matching/TurboFlux/turboflux.h"
#include "matching/matching.h"
#include "utils/globals.h"
#include "utils/types.h"
#ifdef CSM_GPU_PLUGIN
// the engine behind the reference's plugin interface (include/csm_gpu_plugin.h)
#include "csm_gpu_plugin.h"
#endif

// ref_index_access.cpp: the sequential SymBi / TurboFlux index state
bool ref_dump_index(matching* m, const std::string& algo, uint32_t nq, FILE* f, long at);

namespace {

// MurmurHash3 fmix64 finaliser (public domain).
inline uint64_t mix64(uint64_t x) {
  x ^= x >> 33; x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33; return x;
}
inline uint64_t pair_hash(uint32_t q, uint32_t v) {
  return mix64((((uint64_t)(q + 1)) << 32) ^ (uint64_t)v ^ 0x9E3779B97F4A7C15ULL);
}

// Parses embedding lines "m0 m1 ... m{n-1} \n" written by print_enum and
// accumulates sum_over_matches(mix64(sum_q pair_hash(q, m[q]))).
class EnumHashBuf : public std::streambuf {
 public:
  explicit EnumHashBuf(uint32_t nq) : nq_(nq) {}
  uint64_t take() { uint64_t h = acc_; acc_ = 0; cnt_ = 0; return h; }
  uint64_t count() const { return cnt_; }
 protected:
  int overflow(int c) override {
    if (c == EOF) return 0;
    if (c == '\n') { flush_line(); } else { line_.push_back((char)c); }
    return c;
  }
  std::streamsize xsputn(const char* s, std::streamsize n) override {
    for (std::streamsize i = 0; i < n; i++) overflow((unsigned char)s[i]);
    return n;
  }
 private:
  void flush_line() {
    uint64_t s = 0; uint32_t q = 0; bool ok = true;
    const char* p = line_.c_str();
    while (*p) {
      while (*p == ' ') p++;
      if (!*p) break;
      if (*p < '0' || *p > '9') { ok = false; break; }
      uint64_t v = 0;
      while (*p >= '0' && *p <= '9') { v = v * 10 + (uint64_t)(*p - '0'); p++; }
      s += pair_hash(q, (uint32_t)v); q++;
    }
    if (ok && q == nq_) { acc_ += mix64(s); cnt_++; }
    else if (!line_.empty()) { fprintf(stderr, "%s\n", line_.c_str()); }
    line_.clear();
  }
  uint32_t nq_;
  uint64_t acc_ = 0, cnt_ = 0;
  std::string line_;
};

struct Args {
  std::string q, d, u, algo = "graphflow", out, dbin, ubin, dump_index;
  std::string gate;         // after preprocessing: create <gate>.ready, start once <gate>.go exists
  std::vector<long> dump_at;  // update counts after which the index is dumped (0: after preprocessing)
  size_t threads = 1, auto_tuning = 0, max_updates = SIZE_MAX;
  size_t first = 0;         // index of the first stream update to run (the data graph is the state there)
  size_t apply_to = 0;      // apply stream updates [0, N) to the data graph itself, then start at N
  uint64_t max_results = UINT32_MAX;
  double time_budget = 0;   // stop after the update that crosses this many seconds
  double wall_budget = 0;   // hard limit: report and exit even inside an update
  bool homo = false, hash = false;
};

// Completed-update counter shared with the wall-budget watchdog.
std::atomic<size_t> g_done{0};

bool read_binary_graph(const std::string& path, Graph& g) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  char magic[4]; uint32_t ver, n, nvl, nel; uint64_t m;
  if (fread(magic, 1, 4, f) != 4 || memcmp(magic, "CSMG", 4) != 0) { fclose(f); return false; }
  if (fread(&ver, 4, 1, f) != 1 || fread(&n, 4, 1, f) != 1 || fread(&m, 8, 1, f) != 1 ||
      fread(&nvl, 4, 1, f) != 1 || fread(&nel, 4, 1, f) != 1) { fclose(f); return false; }
  std::vector<uint32_t> vl(n), e(3 * m);
  if (fread(vl.data(), 4, n, f) != n || fread(e.data(), 4, 3 * m, f) != 3 * m) { fclose(f); return false; }
  fclose(f);
  for (uint32_t v = 0; v < n; v++) g.AddVertex(v, vl[v]);
  // Sorted (min,max) order makes every Graph::AddEdge an append.
  std::vector<uint64_t> order(m);
  for (uint64_t i = 0; i < m; i++) {
    uint32_t a = std::min(e[3 * i], e[3 * i + 1]), b = std::max(e[3 * i], e[3 * i + 1]);
    order[i] = ((uint64_t)a << 32) | b;
  }
  std::vector<uint64_t> idx(m);
  for (uint64_t i = 0; i < m; i++) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](uint64_t x, uint64_t y) { return order[x] < order[y]; });
  for (uint64_t i : idx) g.AddEdge(e[3 * i], e[3 * i + 1], e[3 * i + 2]);
  return true;
}

bool read_binary_stream(const std::string& path, Graph& g) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  char magic[4]; uint32_t ver; uint64_t n;
  if (fread(magic, 1, 4, f) != 4 || memcmp(magic, "CSMU", 4) != 0) { fclose(f); return false; }
  if (fread(&ver, 4, 1, f) != 1 || fread(&n, 8, 1, f) != 1) { fclose(f); return false; }
  std::vector<uint32_t> rec(4 * n);
  if (fread(rec.data(), 4, 4 * n, f) != 4 * n) { fclose(f); return false; }
  fclose(f);
  g.updates_vec_.clear();
  for (uint64_t i = 0; i < n; i++) {
    uint32_t tw = rec[4 * i];
    char type = (char)(tw & 0xff); bool add = ((tw >> 8) & 0xff) != 0;
    g.updates_.emplace(type, add, rec[4 * i + 1], rec[4 * i + 2], rec[4 * i + 3]);
    g.updates_vec_.emplace_back(type, add, rec[4 * i + 1], rec[4 * i + 2], rec[4 * i + 3]);
  }
  return true;
}

void usage() {
  fprintf(stderr,
          "ref_driver -q query -d data|-D data.bin -u stream|-U stream.bin -a algo\n"
          "  [-t threads] [--auto-tuning 0|1] [--max-results N] [--homo 0|1]\n"
          "  [--hash] [--out per_update.csv] [--max-updates N] [--time-budget S] [--wall-budget S]\n"
          "  [--first N]   (start at stream update N; give the data graph as it stands there)\n"
          "  [--apply-to N] (apply stream updates [0, N) to the data graph with Graph::AddEdge /\n"
          "                 RemoveEdge before preprocessing, then start at update N)\n"
          "  [--gate PATH] (after preprocessing write PATH.ready; start the updates once PATH.go exists)\n"
          "  [--dump-index FILE --dump-at N,N,...]   (symbi / turboflux: root, DAG, d1 / d2 flags)\n");
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  for (int i = 1; i < argc; i++) {
    std::string k = argv[i];
    auto nxt = [&]() -> std::string { if (i + 1 >= argc) { usage(); exit(2); } return argv[++i]; };
    if (k == "-q") a.q = nxt();
    else if (k == "-d") a.d = nxt();
    else if (k == "-D") a.dbin = nxt();
    else if (k == "-u") a.u = nxt();
    else if (k == "-U") a.ubin = nxt();
    else if (k == "-a") a.algo = nxt();
    else if (k == "-t") a.threads = std::stoul(nxt());
    else if (k == "--auto-tuning") a.auto_tuning = std::stoul(nxt());
    else if (k == "--max-results") a.max_results = std::stoull(nxt());
    else if (k == "--homo") a.homo = std::stoi(nxt()) != 0;
    else if (k == "--hash") a.hash = true;
    else if (k == "--out") a.out = nxt();
    else if (k == "--max-updates") a.max_updates = std::stoull(nxt());
    else if (k == "--first") a.first = std::stoull(nxt());
    else if (k == "--apply-to") a.apply_to = std::stoull(nxt());
    else if (k == "--gate") a.gate = nxt();
    else if (k == "--time-budget") a.time_budget = std::stod(nxt());
    else if (k == "--wall-budget") a.wall_budget = std::stod(nxt());
    else if (k == "--dump-index") a.dump_index = nxt();
    else if (k == "--dump-at") {
      std::stringstream ss(nxt());
      std::string t;
      while (std::getline(ss, t, ',')) if (!t.empty()) a.dump_at.push_back(std::stol(t));
    }
    else { usage(); return 2; }
  }
  if (a.q.empty() || (a.d.empty() && a.dbin.empty()) || (a.u.empty() && a.ubin.empty())) { usage(); return 2; }

  auto t0 = std::chrono::steady_clock::now();
  Graph query{}, data{};
  query.LoadFromFile(a.q);
  if (!a.dbin.empty()) { if (!read_binary_graph(a.dbin, data)) { fprintf(stderr, "bad graph %s\n", a.dbin.c_str()); return 1; } }
  else data.LoadFromFile(a.d);
  auto t1 = std::chrono::steady_clock::now();

  // Plugins take `uint max_num_results` (ParaCOSM/CSM/matching/main.cpp:682).
  uint maxr = (uint)std::min<uint64_t>(a.max_results, UINT32_MAX);
  bool print_enum = a.hash;
  std::vector<std::vector<uint>> orders;
  matching* mm = nullptr;
  if (a.algo == "graphflow") mm = new Graphflow(query, data, maxr, false, print_enum, a.homo);
  else if (a.algo == "turboflux") mm = new TurboFlux(query, data, maxr, false, print_enum, a.homo);
  else if (a.algo == "symbi") mm = new SymBi(query, data, maxr, false, print_enum, a.homo, orders);
  else if (a.algo == "parallel_symbi") mm = new Parrllel_SymBi(query, data, maxr, false, print_enum, a.homo, orders, a.threads, a.auto_tuning);
  else if (a.algo == "parallel_turboflux") mm = new Parallel_TurboFlux(query, data, maxr, false, print_enum, a.homo, a.threads, a.auto_tuning);
  else if (a.algo == "parallel_graphflow") mm = new Parallel_Graphflow(query, data, maxr, false, print_enum, a.homo, a.threads, a.auto_tuning);
#ifdef CSM_GPU_PLUGIN
  else if (a.algo == "gpu_graphflow") mm = new GpuPlugin(query, data, maxr, false, print_enum, a.homo, CSM_ALGO_GRAPHFLOW);
  else if (a.algo == "gpu_turboflux") mm = new GpuPlugin(query, data, maxr, false, print_enum, a.homo, CSM_ALGO_TURBOFLUX);
  else if (a.algo == "gpu_symbi") mm = new GpuPlugin(query, data, maxr, false, print_enum, a.homo, CSM_ALGO_SYMBI);
  else if (a.algo == "gpu_calig") mm = new GpuPlugin(query, data, maxr, false, print_enum, a.homo, CSM_ALGO_CALIG);
  else if (a.algo == "gpu_newsp") mm = new GpuPlugin(query, data, maxr, false, print_enum, a.homo, CSM_ALGO_NEWSP);
#endif
  else { fprintf(stderr, "Unknown algorithm %s\n", a.algo.c_str()); return 2; }

  EnumHashBuf hb(query.NumVertices());
  std::streambuf* old = nullptr;
  auto load_stream = [&]() -> bool {
    if (!a.ubin.empty()) return read_binary_stream(a.ubin, data);
    data.LoadUpdateStream(a.u);
    return true;
  };
  if (a.apply_to) {
    // the graph as it stands after the stream's first updates, built by the
    // reference's own Graph methods (no plugin sees these updates)
    if (!load_stream()) { fprintf(stderr, "bad stream\n"); return 1; }
    const size_t na = std::min(a.apply_to, data.updates_vec_.size());
    for (size_t i = 0; i < na; i++) {
      const InsertUnit& up = data.updates_vec_[i];
      if (up.type == 'v' && up.is_add) data.AddVertex(up.id1, up.label);
      else if (up.type == 'v') data.RemoveVertex(up.id1);
      else if (up.is_add) data.AddEdge(up.id1, up.id2, up.label);
      else data.RemoveEdge(up.id1, up.id2);
    }
    a.first = na;
  }
  mm->Preprocessing();
  auto t2 = std::chrono::steady_clock::now();

  if (!a.apply_to && !load_stream()) { fprintf(stderr, "bad stream\n"); return 1; }
  // --first N: the data graph given is the state after updates [0, N), and the
  // loop runs updates N, N + 1, ... in order (rows keep their stream index)
  const size_t first = std::min(a.first, data.updates_vec_.size());
  size_t n_up = data.updates_vec_.size() - first;
  if (a.max_updates < n_up) n_up = a.max_updates;

  FILE* fo = nullptr;
  if (!a.out.empty()) {
    fo = fopen(a.out.c_str(), "w");
    if (!fo) { fprintf(stderr, "cannot write %s\n", a.out.c_str()); return 1; }
    fprintf(fo, "idx,type,is_add,id1,id2,label,pos,neg,latency_ns,hash\n");
  }
  FILE* fdump = nullptr;
  if (!a.dump_index.empty()) {
    fdump = fopen(a.dump_index.c_str(), "w");
    if (!fdump) { fprintf(stderr, "cannot write %s\n", a.dump_index.c_str()); return 1; }
  }
  auto want_dump = [&](long at) { return fdump && std::find(a.dump_at.begin(), a.dump_at.end(), at) != a.dump_at.end(); };
  if (want_dump(0) && !ref_dump_index(mm, a.algo, query.NumVertices(), fdump, 0)) {
    fprintf(stderr, "--dump-index supports symbi and turboflux\n");
    return 2;
  }
  if (!a.gate.empty()) {
    // Several runs can load and preprocess at the same time while their timed
    // update loops are started one after another by whoever holds the gate.
    FILE* fr = fopen((a.gate + ".ready").c_str(), "w");
    if (!fr) { fprintf(stderr, "cannot write %s.ready\n", a.gate.c_str()); return 1; }
    fclose(fr);
    const std::string go = a.gate + ".go";
    auto g0 = std::chrono::steady_clock::now();
    while (access(go.c_str(), F_OK) != 0) {
      if (std::chrono::duration<double>(std::chrono::steady_clock::now() - g0).count() > 7200.0) {
        fprintf(stderr, "gate %s not opened within 7200 s\n", go.c_str());
        return 1;
      }
      std::this_thread::sleep_for(std::chrono::milliseconds(20));
    }
  }
  if (a.hash) old = std::cout.rdbuf(&hb);

  size_t pos_last = 0, neg_last = 0, unsafe = 0, nv = 0, ne = 0, done = 0;
  std::vector<uint64_t> lat(n_up, 0);
  auto ts = std::chrono::steady_clock::now();
  if (a.wall_budget > 0) {
    // Some reference plugins ignore the result cap inside their parallel
    // search, so one update can run for hours: report what finished and exit.
    std::thread([ts, &a, first]() {
      std::this_thread::sleep_for(std::chrono::duration<double>(a.wall_budget));
      double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
      printf("wall_budget_reached updates_done=%zu elapsed_s=%.6f first=%zu\n", g_done.load(), el, first);
      fflush(stdout);
      _exit(0);
    }).detach();
  }
  for (size_t i = 0; i < n_up; i++) {
    const InsertUnit& up = data.updates_vec_[first + i];
    auto s = std::chrono::steady_clock::now();
    if (up.type == 'v' && up.is_add) { mm->AddVertex(up.id1, up.label); nv++; }
    else if (up.type == 'v') { mm->RemoveVertex(up.id1); nv++; }
    else if (up.is_add) { mm->AddEdge(up.id1, up.id2, up.label); ne++; }
    else { mm->RemoveEdge(up.id1, up.id2); ne++; }
    auto e = std::chrono::steady_clock::now();
    lat[i] = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(e - s).count();
    size_t pc = 0, nc = 0;
    mm->GetNumPositiveResults(pc);
    mm->GetNumNegativeResults(nc);
    uint64_t h = a.hash ? hb.take() : 0;
    if (fo) fprintf(fo, "%zu,%c,%d,%u,%u,%u,%zu,%zu,%llu,%llu\n", first + i, up.type, (int)up.is_add, up.id1,
                    up.id2, up.label, pc - pos_last, nc - neg_last, (unsigned long long)lat[i],
                    (unsigned long long)h);
    if (fo) fflush(fo);  // completed updates survive a kill of a run that hangs on a later one
    if (pc != pos_last || nc != neg_last) unsafe++;
    pos_last = pc; neg_last = nc;
    done++;
    if (want_dump((long)done)) { ref_dump_index(mm, a.algo, query.NumVertices(), fdump, (long)done); fflush(fdump); }
    g_done.store(done);
    if (a.time_budget > 0 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count() > a.time_budget)
      break;
  }
  auto te = std::chrono::steady_clock::now();
  if (a.hash) std::cout.rdbuf(old);
  if (fo) fclose(fo);
  if (fdump) fclose(fdump);

  std::vector<uint64_t> l(lat.begin(), lat.begin() + done);
  std::sort(l.begin(), l.end());
  auto pct = [&](double p) -> unsigned long long {
    if (l.empty()) return 0ULL;
    size_t k = (size_t)std::min<double>((double)l.size() - 1, p * (double)(l.size() - 1) + 0.5);
    return (unsigned long long)l[k];
  };
  double inc_s = std::chrono::duration<double>(te - ts).count();
  printf("Load Graphs: %.3f ms\n", std::chrono::duration<double, std::milli>(t1 - t0).count());
  printf("Preprocessing: %.3f ms\n", std::chrono::duration<double, std::milli>(t2 - t1).count());
  printf("Incremental Matching: %.3f ms\n", inc_s * 1e3);
  printf("%zu vertex updates.\n%zu edge updates.\n%zu unsafe updates.\n", nv, ne, unsafe);
  printf("%zu positive matches.\n%zu negative matches.\n", pos_last, neg_last);
  printf("updates_done=%zu elapsed_s=%.6f updates_per_s=%.3f p50_ns=%llu p99_ns=%llu threads=%zu first=%zu\n", done,
         inc_s, done / std::max(inc_s, 1e-12), pct(0.50), pct(0.99), a.threads, first);
  fflush(stdout);
  // Skip destructors of the large hash maps: exit directly.
  _exit(0);
}
