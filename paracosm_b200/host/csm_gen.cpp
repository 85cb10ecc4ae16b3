// csm_gen: writes a seeded synthetic workload (data graph, update stream,
// queries) in the reference's text formats and/or the binary containers.
//
//   csm_gen --preset c1|c2|c3|c4|c5 --out DIR [--seed S] [--text] [--calig] [--no-binary]
//           [--log2-n K] [--avg-degree D] [--vlabels L] [--zipf S] [--elabels L]
//           [--updates N] [--insert-frac F] [--holdout-frac F] [--snapshot-at N]
//           [--query SIZE:dense|sparse[:EXTRA[:MINDEG]]] (repeatable; replaces the preset's)
//
// DIR receives data.bin / stream.bin (binary), data.graph / stream.txt (text,
// with --text), query_<i>.graph, and meta.txt (the spec and sizes).
// --snapshot-at N also writes data_at_<N>.bin: the data graph left by the
// first N updates of the stream, from which a run can start at update N
// (binary only).  --calig
// also writes data.calig / stream.calig / query_<i>.calig in the reference
// CaLiG program's formats (no edge labels; deletions as negative ids).
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "calig_io.h"
#include "workload.h"

using namespace csm;

static void usage() {
  fprintf(stderr,
          "csm_gen --preset c1|c2|c3|c4|c5 --out DIR [--seed S] [--text] [--calig] [--no-binary]\n"
          "        [--log2-n K] [--avg-degree D] [--vlabels L] [--zipf S] [--elabels L]\n"
          "        [--updates N] [--insert-frac F] [--holdout-frac F] [--snapshot-at N]\n"
          "        [--query SIZE:dense|sparse[:EXTRA[:MINDEG]]]...\n");
}

int main(int argc, char** argv) {
  WorkloadSpec s;
  preset("c1", s);
  std::string out;
  bool text = false, calig = false, binary = true, queries_set = false;
  try {  // a malformed number ends the run with the usage text, as an unknown option does
    for (int i = 1; i < argc; i++) {
      std::string k = argv[i];
      auto nxt = [&]() -> std::string { if (i + 1 >= argc) { usage(); exit(2); } return argv[++i]; };
      if (k == "--preset") { if (!preset(nxt(), s)) { fprintf(stderr, "unknown preset\n"); return 2; } }
      else if (k == "--out") out = nxt();
      else if (k == "--seed") s.seed = std::stoull(nxt());
      else if (k == "--text") text = true;
      else if (k == "--calig") calig = true;
      else if (k == "--no-binary") binary = false;
      else if (k == "--log2-n") s.log2_n = (uint32_t)std::stoul(nxt());
      else if (k == "--avg-degree") s.avg_degree = std::stod(nxt());
      else if (k == "--vlabels") s.n_vlabels = (uint32_t)std::stoul(nxt());
      else if (k == "--zipf") s.vlabel_zipf = std::stod(nxt());
      else if (k == "--elabels") s.n_elabels = (uint32_t)std::stoul(nxt());
      else if (k == "--updates") s.n_updates = std::stoull(nxt());
      else if (k == "--insert-frac") s.insert_fraction = std::stod(nxt());
      else if (k == "--holdout-frac") s.holdout_fraction = std::stod(nxt());
      else if (k == "--snapshot-at") s.snapshot_at = std::stoull(nxt());
      else if (k == "--query") {
        if (!queries_set) { s.queries.clear(); queries_set = true; }
        std::string v = nxt();
        QuerySpec q;
        char kind[16] = {0};
        unsigned size = 0, extra = 0; double mindeg = 0;
        int got = sscanf(v.c_str(), "%u:%15[a-z]:%u:%lf", &size, kind, &extra, &mindeg);
        if (got < 2) { usage(); return 2; }
        q.size = size; q.dense = strcmp(kind, "dense") == 0; q.extra_edges = extra; q.min_avg_degree = mindeg;
        s.queries.push_back(q);
      } else { usage(); return 2; }
    }
  } catch (const std::exception&) {
    fprintf(stderr, "bad option value\n");
    usage();
    return 2;
  }
  if (out.empty()) { usage(); return 2; }
  mkdir(out.c_str(), 0755);
  auto t0 = std::chrono::steady_clock::now();
  Workload w;
  std::string err;
  if (!generate(s, w, err)) { fprintf(stderr, "generate: %s\n", err.c_str()); return 1; }
  auto t1 = std::chrono::steady_clock::now();
  bool ok = true;
  if (binary) {
    ok &= save_graph_binary(out + "/data.bin", w.initial);
    ok &= save_stream_binary(out + "/stream.bin", w.stream);
  }
  if (s.snapshot_at)
    ok &= save_graph_binary(out + "/data_at_" + std::to_string(s.snapshot_at) + ".bin", w.snapshot);
  if (text) {
    ok &= save_graph_text(out + "/data.graph", w.initial);
    ok &= save_stream_text(out + "/stream.txt", w.stream);
  }
  for (size_t i = 0; i < w.queries.size(); i++)
    ok &= save_query_text(out + "/query_" + std::to_string(i) + ".graph", w.queries[i]);
  if (calig) {
    ok &= save_calig_graph(out + "/data.calig", w.initial);
    ok &= save_calig_stream(out + "/stream.calig", w.stream);
    for (size_t i = 0; i < w.queries.size(); i++) {
      EdgeList q;
      q.n = w.queries[i].n;
      q.vlabels = w.queries[i].vlabels;
      q.edges = w.queries[i].edges;
      ok &= save_calig_graph(out + "/query_" + std::to_string(i) + ".calig", q);
    }
  }
  FILE* f = fopen((out + "/meta.txt").c_str(), "w");
  if (f) {
    fprintf(f, "name=%s\nseed=%llu\nlog2_n=%u\navg_degree=%g\nrmat=%g,%g,%g\nvlabels=%u\nzipf=%g\nelabels=%u\n",
            s.name.c_str(), (unsigned long long)s.seed, s.log2_n, s.avg_degree, s.rmat_a, s.rmat_b, s.rmat_c,
            s.n_vlabels, s.vlabel_zipf, s.n_elabels);
    fprintf(f, "total_edges=%llu\ninitial_edges=%llu\nupdates=%zu\ninsert_fraction=%g\n",
            (unsigned long long)w.total_edges, (unsigned long long)w.initial.num_edges(), w.stream.size(),
            s.insert_fraction);
    for (size_t i = 0; i < w.queries.size(); i++)
      fprintf(f, "query_%zu=%u vertices %zu edges %s\n", i, w.queries[i].n, w.queries[i].edges.size() / 3,
              s.queries[i].dense ? "dense" : "sparse");
    fclose(f);
  }
  auto t2 = std::chrono::steady_clock::now();
  fprintf(stderr, "generated %s: n=%u initial_edges=%llu updates=%zu queries=%zu in %.2fs (write %.2fs)\n",
          s.name.c_str(), w.initial.n, (unsigned long long)w.initial.num_edges(), w.stream.size(),
          w.queries.size(), std::chrono::duration<double>(t1 - t0).count(),
          std::chrono::duration<double>(t2 - t1).count());
  return ok ? 0 : 1;
}
