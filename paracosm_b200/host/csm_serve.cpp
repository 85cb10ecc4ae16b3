// csm_serve: the serving loop (serve.h) as a command-line tool.
//
//   csm_serve -w WORKLOAD_DIR [--queries N] [--rate R] [--max-batch B] [--budget-gb G]
//             [--cap N] [--plugins symbi,turboflux,graphflow,calig,newsp] [--arrive-every S]
//             [--max-updates N] [--max-seconds S] [--seed S] [--hash 0|1] [--graphs 0|1]
//             [--deadline-ms MS] [--device D] [--rates R1,R2,...]
//             [--out results.bin]
//   csm_serve -d data -u stream -q query[:plugin[:cap[:arrive_s]]] [-q ...] [same options]
//
// A workload directory is the generator's output (data.bin, stream.bin,
// query_<i>.graph); its queries get the plugins round-robin.  Prints one JSON
// line with the offered rate, sustained updates/s, p50 / p99 per-update
// latency (arrival to results on the host), batches and admitted queries.
// --rates sweeps offered loads in one run: --max-seconds of arrivals per
// rate, each segment continuing the stream and the graph where the last one
// stopped; one JSON line per segment ("segment": i) precedes the line of the
// whole run.
// --out writes every admitted query's per-update results:
//   "CSMR", u32 n_queries, then per query: u32 admitted, u64 first, u64 count,
//   count x csm_result (48 bytes).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "graph_io.h"
#include "serve.h"

using namespace csm;

namespace {

int plugin_of(const std::string& s) {
  if (s.find("turboflux") != std::string::npos) return CSM_ALGO_TURBOFLUX;
  if (s.find("symbi") != std::string::npos) return CSM_ALGO_SYMBI;
  if (s.find("graphflow") != std::string::npos) return CSM_ALGO_GRAPHFLOW;
  if (s.find("calig") != std::string::npos) return CSM_ALGO_CALIG;
  if (s.find("newsp") != std::string::npos) return CSM_ALGO_NEWSP;
  return -1;
}

std::vector<std::string> split(const std::string& s, char c) {
  std::vector<std::string> out;
  size_t a = 0;
  while (true) {
    size_t b = s.find(c, a);
    out.push_back(s.substr(a, b == std::string::npos ? std::string::npos : b - a));
    if (b == std::string::npos) break;
    a = b + 1;
  }
  return out;
}

void usage() {
  fprintf(stderr,
          "csm_serve -w DIR | -d data -u stream -q query[:plugin[:cap[:arrive_s]]]...\n"
          "  [--queries N] [--rate R] [--max-batch B] [--budget-gb G] [--cap N] [--plugins a,b,c]\n"
          "  [--arrive-every S] [--max-updates N] [--max-seconds S] [--seed S] [--hash 0|1] [--graphs 0|1]\n"
          "  [--deadline-ms MS] [--device D] [--rates R1,R2,...]\n"
          "  [--out results.bin]\n");
}

}  // namespace

int main(int argc, char** argv) {
  std::string wdir, dpath, upath, out_path;
  std::vector<std::string> qspecs;
  std::vector<std::string> plugins{"parallel_symbi", "parallel_turboflux", "parallel_graphflow"};
  uint64_t cap = 0, max_updates = 0;
  uint32_t nqueries = 0;
  double arrive_every = 0;
  ServeConfig cfg;
  try {  // a malformed number ends the run with the usage text, as an unknown option does
    for (int i = 1; i < argc; i++) {
      const std::string k = argv[i];
      auto val = [&]() -> std::string {
        if (i + 1 >= argc) { usage(); exit(2); }
        return argv[++i];
      };
      if (k == "-w") wdir = val();
      else if (k == "-d") dpath = val();
      else if (k == "-u") upath = val();
      else if (k == "-q") qspecs.push_back(val());
      else if (k == "--queries") nqueries = (uint32_t)std::stoul(val());
      else if (k == "--rate") cfg.rate = std::stod(val());
      else if (k == "--max-batch") cfg.max_batch = (uint32_t)std::stoul(val());
      else if (k == "--budget-gb") cfg.budget_bytes = (uint64_t)(std::stod(val()) * (double)(1ull << 30));
      else if (k == "--cap") cap = std::stoull(val());
      else if (k == "--plugins") plugins = split(val(), ',');
      else if (k == "--arrive-every") arrive_every = std::stod(val());
      else if (k == "--max-updates") max_updates = std::stoull(val());
      else if (k == "--max-seconds") cfg.max_seconds = std::stod(val());
      else if (k == "--seed") cfg.seed = std::stoull(val());
      else if (k == "--hash") cfg.want_hash = std::stoi(val()) != 0;
      else if (k == "--graphs") cfg.graphs = std::stoi(val()) != 0;
      else if (k == "--deadline-ms") cfg.deadline_ns = (uint64_t)(std::stod(val()) * 1e6);
      else if (k == "--device") cfg.device = std::stoi(val());
      else if (k == "--rates") {
        for (const std::string& r : split(val(), ','))
          if (!r.empty()) cfg.rates.push_back(std::stod(r));
      }
      else if (k == "--out") out_path = val();
      else if (k == "-h" || k == "--help") { usage(); return 0; }
      else { fprintf(stderr, "unknown option %s\n", k.c_str()); usage(); return 2; }
    }
  } catch (const std::exception&) {
    fprintf(stderr, "bad option value\n");
    usage();
    return 2;
  }
  EdgeList data;
  std::vector<Update> stream;
  std::vector<ServeQuery> queries;
  std::string err;
  if (!wdir.empty()) {
    dpath = wdir + "/data.bin";
    upath = wdir + "/stream.bin";
    for (uint32_t i = 0; nqueries == 0 || i < nqueries; i++) {
      const std::string qp = wdir + "/query_" + std::to_string(i) + ".graph";
      FILE* f = fopen(qp.c_str(), "r");
      if (!f) break;
      fclose(f);
      qspecs.push_back(qp + ":" + plugins[i % plugins.size()] + ":" + std::to_string(cap) + ":" +
                       std::to_string(arrive_every * i));
    }
  }
  if (dpath.empty() || upath.empty() || qspecs.empty()) { usage(); return 2; }
  if (!load_graph_any(dpath, data, err) || !load_stream_any(upath, stream, err)) {
    fprintf(stderr, "%s\n", err.c_str());
    return 1;
  }
  if (max_updates && stream.size() > max_updates) stream.resize(max_updates);
  for (const std::string& spec : qspecs) {
    std::vector<std::string> p = split(spec, ':');
    EdgeList q;
    if (!load_graph_any(p[0], q, err)) { fprintf(stderr, "%s\n", err.c_str()); return 1; }
    ServeQuery sq;
    sq.vlabels = q.vlabels;
    sq.edges = q.edges;
    sq.algorithm = p.size() > 1 ? plugin_of(p[1]) : CSM_ALGO_GRAPHFLOW;
    if (sq.algorithm < 0) { fprintf(stderr, "unknown plugin in %s\n", spec.c_str()); return 2; }
    sq.max_results = p.size() > 2 && !p[2].empty() ? std::stoull(p[2]) : cap;
    sq.arrive_s = p.size() > 3 && !p[3].empty() ? std::stod(p[3]) : 0.0;
    queries.push_back(sq);
  }
  std::vector<ServeQueryResult> res;
  ServeStats st;
  std::vector<ServeStats> sweep;
  int rc = serve(data, stream, queries, cfg, res, st, err, &sweep);
  if (rc) {
    fprintf(stderr, "serve failed (%d): %s\n", rc, err.c_str());
    return 1;
  }
  if (!cfg.rates.empty()) {
    for (size_t i = 0; i < sweep.size(); i++) {
      const ServeStats& x = sweep[i];
      printf("{\"segment\": %zu, \"offered_rate\": %.1f, \"sustained\": %.1f, \"updates\": %llu, "
             "\"elapsed_s\": %.4f, \"p50_us\": %.1f, \"p99_us\": %.1f, \"batches\": %llu, \"mean_batch\": %.1f, "
             "\"max_batch_seen\": %llu, \"queries_admitted\": %u, \"queries_refused\": %u, "
             "\"device_bytes\": %llu, \"success_rate\": %.6f}\n",
             i, cfg.rates[i], x.sustained, (unsigned long long)x.updates, x.elapsed_s, x.p50_us, x.p99_us,
             (unsigned long long)x.batches, x.mean_batch, (unsigned long long)x.max_batch_seen, x.queries_admitted,
             x.queries_refused, (unsigned long long)x.device_bytes,
             x.results ? 1.0 - (double)x.incomplete / (double)x.results : 1.0);
    }
  }
  uint64_t pos = 0, neg = 0, capped = 0;
  for (const ServeQueryResult& r : res)
    for (const csm_result& x : r.results) { pos += x.pos; neg += x.neg; capped += x.status == CSM_ST_CAPPED; }
  printf("{\"offered_rate\": %.1f, \"sustained\": %.1f, \"updates\": %llu, \"elapsed_s\": %.4f, \"p50_us\": %.1f, "
         "\"p99_us\": %.1f, \"batches\": %llu, \"mean_batch\": %.1f, \"max_batch_seen\": %llu, "
         "\"queries\": %zu, \"queries_admitted\": %u, \"queries_refused\": %u, \"device_bytes\": %llu, "
         "\"positive\": %llu, \"negative\": %llu, \"capped\": %llu, \"success_rate\": %.6f}\n",
         cfg.rate, st.sustained, (unsigned long long)st.updates, st.elapsed_s, st.p50_us, st.p99_us,
         (unsigned long long)st.batches, st.mean_batch, (unsigned long long)st.max_batch_seen, queries.size(),
         st.queries_admitted, st.queries_refused, (unsigned long long)st.device_bytes, (unsigned long long)pos,
         (unsigned long long)neg, (unsigned long long)capped,
         st.results ? 1.0 - (double)st.incomplete / (double)st.results : 1.0);
  if (!out_path.empty()) {
    FILE* f = fopen(out_path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", out_path.c_str()); return 1; }
    const uint32_t nq = (uint32_t)res.size();
    fwrite("CSMR", 1, 4, f);
    fwrite(&nq, 4, 1, f);
    for (const ServeQueryResult& r : res) {
      const uint32_t adm = r.admitted ? 1 : 0;
      const uint64_t first = r.first, cnt = r.results.size();
      fwrite(&adm, 4, 1, f);
      fwrite(&first, 8, 1, f);
      fwrite(&cnt, 8, 1, f);
      if (cnt) fwrite(r.results.data(), sizeof(csm_result), cnt, f);
    }
    fclose(f);
  }
  return 0;
}
