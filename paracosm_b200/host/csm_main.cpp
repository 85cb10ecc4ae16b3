// csm: the reference's command-line driver (ParaCOSM/CSM/matching/main.cpp:676-871)
// over the CUDA engine.
//
//   csm -q query.graph -d data.graph -u stream.txt -a parallel_symbi
//       [--max-results N] [--time-limit S] [--print-prep 0|1] [--print-enum 0|1]
//       [--homo 0|1] [--report-initial 0|1] [--initial-time-limit S] [--orders ...]
//       [-t N] [--auto-tuning 0|1]
//     engine options (not in the reference):
//       [--mode batched|plain] [--batch N] [--device N] [--hash 0|1]
//       [--turboflux-compat 0|1] [--out per_update.csv]
//
// Prints the reference's sections and summary lines.  The update stream is
// processed with the sequential semantics of SingleThreadUpdate
// (main.cpp:628-674: every update applied and counted in stream order), not
// with the shipped BatchUpdates3 (main.cpp:253-397), which skips updates.
// -t / --auto-tuning pick CPU thread counts in the reference; here -t is
// accepted and ignored, and --auto-tuning 1 lets the engine choose its
// launch shape.  --print-enum 1 prints every embedding as the reference does
// ("m0 m1 ... " per line, SymBi/symbi.cpp:564-569), grouped by update, in an
// unspecified order inside an update; --hash 1 and --out give per-update
// counts and match-set hashes without printing.  --orders is accepted and
// ignored (the engine derives its own orders).
// Files may also be the generator's binary CSMG / CSMU containers.
//
// -q may name a directory: every file in it (names not starting with '.',
// in name order) is a query on the same data graph, as in NewSP's
// multi-query build (ParaCOSM/CSM/matching/Parallel_NewSP/graph/graph.cpp:550-574).
// The first is the plugin's own query, the others are attached as standing
// queries with the same plugin and cap; each update's counts are summed over
// all queries.  --print-enum and the per-update hash cover the first query.
#include <dirent.h>
#include <sys/resource.h>
#include <sys/stat.h>

#include <algorithm>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "graph_io.h"
#include "plugins.h"

using namespace csm;

namespace {

using Clock = std::chrono::high_resolution_clock;

double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

bool parse_bool(const std::string& v) { return v == "1" || v == "true" || v == "on" || v == "yes"; }

long peak_vm_kb() {
  std::ifstream f("/proc/self/status");
  std::string line;
  while (std::getline(f, line))
    if (line.rfind("VmPeak:", 0) == 0) return std::strtol(line.c_str() + 7, nullptr, 10);
  return 0;
}

void usage() {
  fprintf(stderr,
          "csm -q query -d data -u stream [-a algorithm] [--max-results N] [--time-limit S]\n"
          "    [--print-prep 0|1] [--print-enum 0|1] [--homo 0|1] [--report-initial 0|1]\n"
          "    [--initial-time-limit S] [--orders ...] [-t N] [--auto-tuning 0|1]\n"
          "    [--mode batched|plain] [--batch N] [--device N] [--hash 0|1] [--turboflux-compat 0|1]\n"
          "    [--out per_update.csv]\n"
          "algorithms: parallel_graphflow parallel_turboflux parallel_symbi parallel_calig parallel_newsp\n"
          "            (graphflow turboflux symbi calig newsp alias them)\n");
}

}  // namespace

int main(int argc, char** argv) {
  std::string query_path, initial_path, stream_path, algorithm = "none", out_path;
  uint64_t max_num_results = 0xffffffffull;
  double time_limit = 0, initial_time_limit = 0;
  bool print_prep = true, print_enum = false, homo = false, report_initial = true;
  size_t thread_num = 6, auto_tuning = 1;
  GpuOptions opt;
  try {  // a malformed number ends the run with the usage text, as an unknown option does
    for (int i = 1; i < argc; i++) {
      const std::string k = argv[i];
      auto val = [&]() -> std::string {
        if (i + 1 >= argc) { usage(); exit(2); }
        return argv[++i];
      };
      if (k == "-q" || k == "--query") query_path = val();
      else if (k == "-d" || k == "--data") initial_path = val();
      else if (k == "-u" || k == "--update") stream_path = val();
      else if (k == "-a" || k == "--algorithm") algorithm = val();
      else if (k == "--max-results") max_num_results = std::stoull(val());
      else if (k == "--time-limit") time_limit = std::stod(val());
      else if (k == "--print-prep") print_prep = parse_bool(val());
      else if (k == "--print-enum") print_enum = parse_bool(val());
      else if (k == "--homo") homo = parse_bool(val());
      else if (k == "--report-initial") report_initial = parse_bool(val());
      else if (k == "--initial-time-limit") initial_time_limit = std::stod(val());
      else if (k == "--orders") { while (i + 1 < argc && argv[i + 1][0] != '-') i++; }
      else if (k == "-t" || k == "--thread-num") thread_num = std::stoul(val());
      else if (k == "--auto-tuning") auto_tuning = std::stoul(val());
      else if (k == "--mode") opt.mode = val() == "plain" ? CSM_MODE_PLAIN : CSM_MODE_BATCHED;
      else if (k == "--batch") opt.max_batch = (uint32_t)std::stoul(val());
      else if (k == "--device") opt.device = std::stoi(val());
      else if (k == "--hash") opt.want_hash = parse_bool(val());
      else if (k == "--turboflux-compat") opt.turboflux_compat = parse_bool(val());
      else if (k == "--out") out_path = val();
      else if (k == "-h" || k == "--help") { usage(); return 0; }
      else { fprintf(stderr, "unknown option %s\n", k.c_str()); usage(); return 2; }
    }
  } catch (const std::exception&) {
    fprintf(stderr, "bad option value\n");
    usage();
    return 2;
  }
  if (query_path.empty() || initial_path.empty() || stream_path.empty()) {
    fprintf(stderr, "-q, -d and -u are required\n");
    usage();
    return 2;
  }
  (void)thread_num;
  (void)initial_time_limit;
  if (print_enum) {
    opt.enum_capacity = 1u << 24;  // embeddings kept per chunk of the stream
    opt.graphs = false;
  }

  auto start = Clock::now();
  printf("----------- Loading graphs ------------\n");
  EdgeList query, data;
  std::string err;
  struct stat qs;
  if (stat(query_path.c_str(), &qs) == 0 && S_ISDIR(qs.st_mode)) {
    std::vector<std::string> names;
    if (DIR* dir = opendir(query_path.c_str())) {
      while (dirent* e = readdir(dir))
        if (e->d_name[0] != '.') names.push_back(query_path + "/" + e->d_name);
      closedir(dir);
    }
    std::sort(names.begin(), names.end());
    if (names.empty()) { printf("no query files in %s\n", query_path.c_str()); return 1; }
    for (size_t i = 0; i < names.size(); i++) {
      EdgeList q;
      if (!load_graph_any(names[i], q, err)) { printf("%s\n", err.c_str()); return 1; }
      if (i == 0) query = q;
      else opt.more_queries.push_back(q);
    }
    printf("Load query graph number: %zu\n", names.size());
  } else if (!load_graph_any(query_path, query, err)) {
    printf("%s\n", err.c_str());
    return 1;
  }
  printf("# vertices = %u\n# edges = %llu\n", query.n, (unsigned long long)query.num_edges());
  if (!load_graph_any(initial_path, data, err)) { printf("%s\n", err.c_str()); return 1; }
  printf("# vertices = %u\n# edges = %llu\n", data.n, (unsigned long long)data.num_edges());
  printf("Load Graphs: %.3fms\n", ms_since(start));

  printf("------------ Preprocessing ------------\n");
  start = Clock::now();
  if (auto_tuning == 0 && opt.warps_per_block == 0) opt.warps_per_block = 8;
  std::unique_ptr<matching> mm(make_plugin(algorithm, query, data, max_num_results, print_prep, print_enum, homo, opt));
  if (!mm) {
    printf("Unknown algorithm\n");
    return 1;
  }
  mm->Preprocessing();
  if (mm->error()) { printf("error: %s\n", mm->error_text().c_str()); return 1; }
  printf("Preprocessing: %.3fms\n", ms_since(start));

  if (report_initial) {
    printf("----------- Initial Matching ----------\n");
    start = Clock::now();
    mm->InitialMatching();
    if (mm->error()) { printf("error: %s\n", mm->error_text().c_str()); return 1; }
    printf("Initial Matching: %.3fms\n", ms_since(start));
    size_t n = 0;
    mm->GetNumInitialResults(n);
    printf("%zu matches. \n", n);
  }

  printf("--------- Incremental Matching --------\n");
  if (auto_tuning == 1) printf("auto_tuning on:%zu\n", auto_tuning);
  else printf("auto_tuning off:%zu\n", auto_tuning);
  std::vector<Update> stream;
  if (!load_stream_any(stream_path, stream, err)) { printf("%s\n", err.c_str()); return 1; }
  size_t num_v = 0, num_e = 0, unsafe = 0, done = 0;
  std::vector<csm_result> res;
  std::vector<csm_result> all;
  if (!out_path.empty()) all.reserve(stream.size());
  start = Clock::now();
  // chunks of the stream: the time limit is checked between chunks
  const size_t chunk = opt.mode == CSM_MODE_PLAIN ? 256 : std::max<size_t>(opt.max_batch, 1) * 4;
  for (size_t a = 0; a < stream.size(); a += chunk) {
    const size_t b = std::min(stream.size(), a + chunk);
    std::vector<Update> part(stream.begin() + (long)a, stream.begin() + (long)b);
    if (mm->ProcessUpdates(part, res)) break;
    if (print_enum && mm->PrintMatches(part.size()) != CSM_OK) break;
    for (size_t i = 0; i < part.size(); i++) {
      if (part[i].type == 'v') num_v++; else num_e++;
      if (res[i].pos || res[i].neg) unsafe++;
    }
    if (!out_path.empty()) all.insert(all.end(), res.begin(), res.end());
    done = b;
    if (time_limit > 0 && ms_since(start) > time_limit * 1e3) break;
  }
  const double inc_ms = ms_since(start);
  if (mm->error()) { printf("error: %s\n", mm->error_text().c_str()); return 1; }
  printf("Incremental Matching: %.3fms\n", inc_ms);
  printf("%zu vertex updates.\n%zu edge updates.\n%zu unsafe updates.\n", num_v, num_e, unsafe);
  size_t pos = 0, neg = 0;
  mm->GetNumPositiveResults(pos);
  mm->GetNumNegativeResults(neg);
  printf("%zu positive matches.\n%zu negative matches.\n", pos, neg);
  mm->PrintCounter();
  size_t ie = 0, iv = 0;
  mm->GetMemoryCost(ie, iv);
  printf("\n# edges in index in total: %zu", ie);
  printf("\n# vertices in index in total: %zu", iv);
  printf("\nPeak Virtual Memory: %ld KB", peak_vm_kb());
  printf("\n\n----------------- End -----------------\n");
  if (!out_path.empty()) {
    FILE* f = fopen(out_path.c_str(), "w");
    if (!f) { fprintf(stderr, "cannot write %s\n", out_path.c_str()); return 1; }
    fprintf(f, "idx,type,is_add,id1,id2,label,pos,neg,latency_ns,hash,status\n");
    for (size_t i = 0; i < done && i < all.size(); i++) {
      const Update& u = stream[i];
      const csm_result& r = all[i];
      fprintf(f, "%zu,%c,%d,%u,%u,%u,%llu,%llu,%llu,%llu,%u\n", i, u.type, (int)u.is_add, u.id1, u.id2, u.label,
              (unsigned long long)r.pos, (unsigned long long)r.neg, (unsigned long long)r.latency_ns,
              (unsigned long long)r.hash, r.status);
    }
    fclose(f);
  }
  return 0;
}
