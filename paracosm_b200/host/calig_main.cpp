// calig: the reference's CaLiG program (ParaCOSM/CSM/matching/Parallel_CaLiG/
// parallel_calig.cpp:1414-1481) over the CUDA engine.
//
//   calig -d data -q query -s stream [-c max_updates] [-t threads]
//     engine options (not in the reference):
//       [--compat 0|1] [--mode batched|plain] [--batch N] [--device N]
//       [--max-results N] [--out per_update.csv] [--skip-mask FILE]
//
// Reads CaLiG's formats (calig_io.h) and prints the reference's progress
// lines and totals on stderr ("added matches: N", "deleted matches: N",
// "updated matches: N", ...).  -t selects CPU threads in the reference; it
// is accepted, and only picks which of the reference's two banner lines is
// printed.
//
// --compat 1 (the default) reproduces two behaviours of the reference's
// update loop: insertions it skips as "safe" count 0 and their edges are
// never searched (calig_skipped_insertions), and each update's count is an
// unsigned 32-bit value (numAdd / searchCore return uint, :1014, :1062).
// --compat 0 counts every insertion exactly.  Deletion records, which the
// reference reads but cannot process (it compares an unsigned id with 0,
// :1228), are processed here: each counts the embeddings it destroys, before
// removing the edge.  --skip-mask FILE writes the --compat skip decision of
// each update (one 0/1 per line) and exits without using the GPU.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "calig_io.h"
#include "plugins.h"

using namespace csm;

namespace {

using Clock = std::chrono::high_resolution_clock;

double ms_since(Clock::time_point t0) { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

void usage() {
  fprintf(stderr,
          "calig -d data -q query -s stream [-c max_updates] [-t threads]\n"
          "      [--compat 0|1] [--mode batched|plain] [--batch N] [--device N] [--max-results N]\n"
          "      [--out per_update.csv] [--skip-mask FILE]\n");
}

}  // namespace

int main(int argc, char** argv) {
  std::string g_path, q_path, s_path, out_path, mask_path;
  uint64_t cnum = 0, max_results = 0;
  size_t thread_num = 32;
  bool compat = true;
  GpuOptions opt;
  try {  // a malformed number ends the run with the usage text, as an unknown option does
    for (int i = 1; i < argc; i++) {
      const std::string k = argv[i];
      auto val = [&]() -> std::string {
        if (i + 1 >= argc) { usage(); exit(2); }
        return argv[++i];
      };
      if (k == "-d") g_path = val();
      else if (k == "-q") q_path = val();
      else if (k == "-s") s_path = val();
      else if (k == "-c") cnum = std::stoull(val());
      else if (k == "-t") thread_num = std::stoul(val());
      else if (k == "--compat") compat = val() != "0";
      else if (k == "--mode") opt.mode = val() == "plain" ? CSM_MODE_PLAIN : CSM_MODE_BATCHED;
      else if (k == "--batch") opt.max_batch = (uint32_t)std::stoul(val());
      else if (k == "--device") opt.device = std::stoi(val());
      else if (k == "--max-results") max_results = std::stoull(val());
      else if (k == "--out") out_path = val();
      else if (k == "--skip-mask") mask_path = val();
      else if (k == "-h" || k == "--help") { usage(); return 0; }
      else { fprintf(stderr, "unknown option %s\n", k.c_str()); usage(); return 2; }
    }
  } catch (const std::exception&) {
    fprintf(stderr, "bad option value\n");
    usage();
    return 2;
  }
  if (g_path.empty() || q_path.empty() || s_path.empty()) { usage(); return 2; }

  auto t0 = Clock::now();
  fprintf(stderr, "========== Start inputting. ==========\n");
  EdgeList query, data;
  std::vector<Update> stream;
  std::string err;
  if (!load_calig_graph(q_path, query, err) || !load_calig_graph(g_path, data, err) ||
      !load_calig_stream(s_path, stream, err, cnum)) {
    fprintf(stderr, "%s\n", err.c_str());
    return 1;
  }
  fprintf(stderr, "Inputting cost (ms): %.3f\n", ms_since(t0));
  fprintf(stderr, "The number of vertices in Q: %u\n", query.n);
  fprintf(stderr, "The number of vertices in G: %u\n", data.n);
  fprintf(stderr, "========== End inputting. ==========\n");
  if (!mask_path.empty()) {
    const std::vector<uint8_t> m = calig_skipped_insertions(query, data, stream);
    FILE* f = fopen(mask_path.c_str(), "w");
    if (!f) { fprintf(stderr, "cannot write %s\n", mask_path.c_str()); return 1; }
    for (uint8_t b : m) fprintf(f, "%d\n", (int)b);
    return fclose(f) == 0 ? 0 : 1;
  }

  // constructCand + staticFilter: the engine's graph and lighting filter
  t0 = Clock::now();
  fprintf(stderr, "========== Start constructing. ==========\n");
  std::unique_ptr<matching> mm(
      make_plugin("parallel_calig", query, data, max_results ? max_results : 0xffffffffull, false, false, false, opt));
  mm->Preprocessing();
  if (mm->error()) { fprintf(stderr, "error: %s\n", mm->error_text().c_str()); return 1; }
  fprintf(stderr, "Constructing cost (ms): %.3f\n", ms_since(t0));
  fprintf(stderr, "========== End constructing. ==========\n");
  fprintf(stderr, "========== Start static filtering. ==========\n");
  fprintf(stderr, "Static filtering cost (ms): %.3f\n", 0.0);
  fprintf(stderr, "========== End static filtering. ==========\n");

  const std::vector<uint8_t> skip = compat ? calig_skipped_insertions(query, data, stream)
                                           : std::vector<uint8_t>(stream.size(), 0);
  std::vector<Update> run;
  std::vector<size_t> where;  // index in `stream` of each submitted update
  for (size_t i = 0; i < stream.size(); i++)
    if (!skip[i]) { run.push_back(stream[i]); where.push_back(i); }

  if (thread_num == 1) fprintf(stderr, "========== Start updating for single thread ==========\n");
  else fprintf(stderr, "========== Start updating for %zu thread ==========\n", thread_num);
  t0 = Clock::now();
  std::vector<csm_result> res;
  if (!run.empty() && mm->ProcessUpdates(run, res)) {
    fprintf(stderr, "error: %s\n", mm->error_text().c_str());
    return 1;
  }
  const double upd_ms = ms_since(t0);
  std::vector<uint64_t> pos(stream.size(), 0), neg(stream.size(), 0);
  for (size_t j = 0; j < run.size(); j++) {
    pos[where[j]] = compat ? (uint32_t)res[j].pos : res[j].pos;
    neg[where[j]] = compat ? (uint32_t)res[j].neg : res[j].neg;
  }
  unsigned long long added = 0, deleted = 0;
  for (size_t i = 0; i < stream.size(); i++) { added += pos[i]; deleted += neg[i]; }
  fprintf(stderr, "added matches: %llu\n", added);
  fprintf(stderr, "deleted matches: %llu\n", deleted);
  fprintf(stderr, "Auxiliary Data Structure update time: %.3fms\n", 0.0);
  fprintf(stderr, "updated matches: %llu\n", added + deleted);
  fprintf(stderr, "search time: %.3fms\n", upd_ms);
  fprintf(stderr, "Updating totally cost (ms): %.3f\n", upd_ms);
  if (thread_num == 1) fprintf(stderr, "========== End single thread updating. ==========\n");
  else fprintf(stderr, "========== End Multi tgihread updating. ==========\n\n========== DONE!! ==========\n");

  if (!out_path.empty()) {
    FILE* f = fopen(out_path.c_str(), "w");
    if (!f) { fprintf(stderr, "cannot write %s\n", out_path.c_str()); return 1; }
    fprintf(f, "idx,is_add,id1,id2,pos,neg,skipped\n");
    for (size_t i = 0; i < stream.size(); i++)
      fprintf(f, "%zu,%d,%u,%u,%llu,%llu,%d\n", i, (int)stream[i].is_add, stream[i].id1, stream[i].id2,
              (unsigned long long)pos[i], (unsigned long long)neg[i], (int)skip[i]);
    fclose(f);
  }
  return 0;
}
