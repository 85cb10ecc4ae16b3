// Per-update driver over the reference's CaLiG plugin
// (ParaCOSM/CSM/matching/Parallel_CaLiG/parallel_calig.cpp), compiled from
// that source file where it lies, with its OpenMP pragmas inactive (no
// -fopenmp: every loop runs serially, so the result does not depend on the
// thread schedule).  Test infrastructure only.
//
//   calig_ref -d data -q query -s stream [--out per_update.txt] [--dump-li li.txt]
//
// The file formats are CaLiG's own (matching/CaLiG/README.md): `v id label`,
// `e a b` without edge labels; a stream of `e a b` insertions.  The
// reference reads stream ids as unsigned integers, so its deletion records
// (`e -a-1 -b-1`) never reach its deletion branch (parallel_calig.cpp:1228
// tests `v1 < 0` on an unsigned value); such records are refused here.
//
// The update loop is the insertion branch of updateAndMatching
// (parallel_calig.cpp:1214-1272), with the count of each update written out
// instead of summed: an update whose endpoint has a label the query does not
// use, an edge already present, or one that turnOnProcess_safe classifies as
// safe counts 0; otherwise the lighting index is updated
// (turnOnProcess_safe_parallel) and searchMatch counts the new embeddings.
//
// --dump-li writes the lighting state after static filtering (constructCand +
// staticFilter, :337-361 and :970-975): one `u v` line per lit pair, sorted.
#include <algorithm>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#define main calig_reference_main
#include CALIG_SRC
#undef main

int main(int argc, char** argv) {
  std::string gp, qp, sp, out_path, li_path;
  for (int i = 1; i + 1 < argc; i++) {
    const std::string k = argv[i];
    if (k == "-d") gp = argv[++i];
    else if (k == "-q") qp = argv[++i];
    else if (k == "-s") sp = argv[++i];
    else if (k == "--out") out_path = argv[++i];
    else if (k == "--dump-li") li_path = argv[++i];
  }
  if (gp.empty() || qp.empty() || sp.empty()) {
    fprintf(stderr, "usage: calig_ref -d data -q query -s stream [--out f] [--dump-li f]\n");
    return 2;
  }
  inputQ(qp);
  generateMO();
  inputG(gp);
  inputUpdate(sp, 0);
  constructCand();
  staticFilter();
  if (!li_path.empty()) {
    std::vector<std::pair<uint, uint>> lit;
    for (uint v = 0; v < G_size; v++)
      for (auto& li : G[v].LI)
        if (li.second) lit.emplace_back(li.first, v);
    std::sort(lit.begin(), lit.end());
    FILE* f = fopen(li_path.c_str(), "w");
    if (!f) return 1;
    for (auto& p : lit) fprintf(f, "%u %u\n", p.first, p.second);
    fclose(f);
  }
  FILE* out = out_path.empty() ? stdout : fopen(out_path.c_str(), "w");
  if (!out) return 1;
  unsigned long long total = 0;
  for (size_t t = 0; t + 1 < update.size(); t += 2) {
    uint v1 = update[t], v2 = update[t + 1];
    if (v1 >= G_size || v2 >= G_size) {
      fprintf(stderr, "update %zu: id out of range (deletion records are not handled by the reference)\n", t / 2);
      return 3;
    }
    uint count = 0;
    if (G[v1].label == (uint)-1 || G[v2].label == (uint)-1) {
    } else if (G[v1].nei.count(v2)) {
    } else if (turnOnProcess_safe(v1, v2)) {
    } else {
      turnOnProcess_safe_parallel(v1, v2);
      count = searchMatch(v1, v2);
    }
    total += count;
    fprintf(out, "%u\n", count);
  }
  if (out != stdout) fclose(out);
  fprintf(stderr, "added matches: %llu\n", total);
  return 0;
}
