// Serving loop (see serve.h).
#include "serve.h"

#include <algorithm>
#include <chrono>
#include <random>
#include <thread>

namespace csm {

namespace {

using Clock = std::chrono::steady_clock;

struct Ctx {
  csm_ctx* h = nullptr;
  ~Ctx() { if (h) csm_gpu_destroy(h); }
};

int fail(int rc, std::string& err, const char* what) {
  const char* t = csm_gpu_last_error();
  err = std::string(what) + ": " + (t ? t : "");
  return rc;
}

uint64_t device_bytes(csm_ctx* c) {
  csm_stats s;
  return csm_gpu_stats(c, &s) == CSM_OK ? s.device_bytes : 0;
}

}  // namespace

int serve(const EdgeList& data, const std::vector<Update>& stream, const std::vector<ServeQuery>& queries,
          const ServeConfig& cfg, std::vector<ServeQueryResult>& out, ServeStats& stats, std::string& err,
          std::vector<ServeStats>* sweep) {
  stats = ServeStats{};
  if (sweep) sweep->clear();
  out.assign(queries.size(), ServeQueryResult{});
  if (queries.empty()) { err = "no query"; return CSM_EINVAL; }
  // the owner context holds the graph and the first query
  const ServeQuery& q0 = queries[0];
  csm_cfg c;
  csm_gpu_default_cfg(&c);
  c.algorithm = q0.algorithm;
  c.max_results = q0.max_results;
  c.max_batch = cfg.max_batch;
  c.want_hash = cfg.want_hash ? 1 : 0;
  c.device = cfg.device;
  c.graphs = cfg.graphs ? CSM_GRAPHS_ON : CSM_GRAPHS_OFF;
  c.deadline_ns = cfg.deadline_ns;  // attached queries inherit it
  Ctx owner;
  int rc = csm_gpu_create(&c, &owner.h);
  if (rc) return fail(rc, err, "create");
  rc = csm_gpu_set_query(owner.h, (uint32_t)q0.vlabels.size(), q0.vlabels.data(), (uint32_t)(q0.edges.size() / 3),
                         q0.edges.data());
  if (rc) return fail(rc, err, "query 0");
  {  // every label a later query may use stays distinct in the shared graph
    std::vector<uint32_t> vl, el;
    for (const ServeQuery& q : queries) {
      vl.insert(vl.end(), q.vlabels.begin(), q.vlabels.end());
      for (size_t i = 2; i < q.edges.size(); i += 3) el.push_back(q.edges[i]);
    }
    rc = csm_gpu_reserve_labels(owner.h, (uint32_t)vl.size(), vl.data(), (uint32_t)el.size(), el.data());
    if (rc) return fail(rc, err, "labels");
  }
  rc = csm_gpu_load_graph(owner.h, data.n, data.vlabels.data(), data.num_edges(), data.edges.data());
  if (!rc) rc = csm_gpu_build_index(owner.h);
  if (rc) return fail(rc, err, "graph");
  out[0].admitted = true;
  std::vector<Ctx> att(queries.size());
  std::vector<size_t> order;  // later queries by arrival time
  for (size_t k = 1; k < queries.size(); k++) order.push_back(k);
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return queries[a].arrive_s < queries[b].arrive_s; });
  size_t next_q = 0;
  uint64_t used = device_bytes(owner.h);

  // Poisson arrivals of the updates, segment by segment (one per offered rate)
  const size_t n = stream.size();
  const std::vector<double> rates = cfg.rates.empty() ? std::vector<double>{cfg.rate} : cfg.rates;
  std::vector<double> lat_all;
  std::vector<csm_result> tmp;
  const auto t_run = Clock::now();
  size_t next = 0;
  for (size_t seg = 0; seg < rates.size() && next < n; seg++) {
    ServeStats ss{};
    const double rate = rates[seg] > 0 ? rates[seg] : 1.0;
    const size_t seg_first = next;
    std::vector<double> arr(n - seg_first);
    {
      std::mt19937_64 rng(cfg.seed + seg);
      std::exponential_distribution<double> gap(rate);
      double t = 0;
      for (size_t i = 0; i < arr.size(); i++) { t += gap(rng); arr[i] = t; }
    }
    std::vector<double> lat;
    const auto t0 = Clock::now();
    auto now_s = [&]() { return std::chrono::duration<double>(Clock::now() - t0).count(); };
    // query arrival times count from the start of the run
    const double seg_start = std::chrono::duration<double>(t0 - t_run).count();
    while (next < n) {
      double t = now_s();
      if (cfg.max_seconds > 0 && t > cfg.max_seconds) break;
      // standing queries that have arrived
      while (next_q < order.size() && queries[order[next_q]].arrive_s <= seg_start + t) {
        const size_t k = order[next_q++];
        const ServeQuery& q = queries[k];
        csm_cfg qc;
        csm_gpu_default_cfg(&qc);
        qc.algorithm = q.algorithm;
        qc.max_results = q.max_results;
        qc.want_hash = cfg.want_hash ? 1 : 0;
        rc = csm_gpu_attach_query(owner.h, &qc, (uint32_t)q.vlabels.size(), q.vlabels.data(),
                                  (uint32_t)(q.edges.size() / 3), q.edges.data(), &att[k].h);
        if (rc == CSM_ENOMEM) { stats.queries_refused++; continue; }
        if (rc) return fail(rc, err, "attach");
        const uint64_t b = device_bytes(att[k].h);
        if (used + b > cfg.budget_bytes) {  // does not fit the budget: refused
          csm_gpu_destroy(att[k].h);
          att[k].h = nullptr;
          stats.queries_refused++;
          continue;
        }
        used += b;
        out[k].admitted = true;
        out[k].first = next;
      }
      // updates that have arrived
      const size_t avail = seg_first + (size_t)(std::upper_bound(arr.begin(), arr.end(), t) - arr.begin());
      if (avail <= next) {
        double wake = arr[next - seg_first];
        if (next_q < order.size()) wake = std::min(wake, queries[order[next_q]].arrive_s - seg_start);
        const double dt = wake - now_s();
        if (dt > 50e-6) std::this_thread::sleep_for(std::chrono::duration<double>(dt - 20e-6));
        continue;
      }
      const size_t B = std::min<size_t>(avail - next, cfg.max_batch);
      rc = csm_gpu_submit(owner.h, B, reinterpret_cast<const csm_update*>(stream.data() + next));
      if (!rc) rc = csm_gpu_wait(owner.h, 0);
      if (rc) return fail(rc, err, "submit");
      for (size_t k = 0; k < queries.size(); k++) {
        csm_ctx* h = k == 0 ? owner.h : att[k].h;
        if (!h) continue;
        tmp.resize(B);
        rc = csm_gpu_results(h, next, B, tmp.data());
        if (rc) return fail(rc, err, "results");
        out[k].results.insert(out[k].results.end(), tmp.begin(), tmp.end());
        for (const csm_result& x : tmp) {
          ss.results++;
          if (x.status == CSM_ST_CAPPED || x.status == CSM_ST_TIMED_OUT) ss.incomplete++;
        }
      }
      const double done = now_s();
      for (size_t i = next; i < next + B; i++) lat.push_back(done - arr[i - seg_first]);
      next += B;
      ss.batches++;
      ss.max_batch_seen = std::max<uint64_t>(ss.max_batch_seen, B);
    }
    ss.elapsed_s = now_s();
    ss.updates = next - seg_first;
    ss.sustained = ss.elapsed_s > 0 ? (double)ss.updates / ss.elapsed_s : 0;
    ss.mean_batch = ss.batches ? (double)ss.updates / (double)ss.batches : 0;
    if (!lat.empty()) {
      std::vector<double> srt = lat;
      std::sort(srt.begin(), srt.end());
      auto pct = [&](double p) { return srt[std::min(srt.size() - 1, (size_t)(p * (double)(srt.size() - 1) + 0.5))]; };
      ss.p50_us = pct(0.50) * 1e6;
      ss.p99_us = pct(0.99) * 1e6;
    }
    ss.device_bytes = used;
    for (const ServeQueryResult& r : out) ss.queries_admitted += r.admitted ? 1 : 0;
    ss.queries_refused = stats.queries_refused;
    if (sweep) sweep->push_back(ss);
    lat_all.insert(lat_all.end(), lat.begin(), lat.end());
    stats.batches += ss.batches;
    stats.max_batch_seen = std::max(stats.max_batch_seen, ss.max_batch_seen);
    stats.elapsed_s += ss.elapsed_s;
  }
  stats.updates = next;
  stats.sustained = stats.elapsed_s > 0 ? (double)next / stats.elapsed_s : 0;
  stats.mean_batch = stats.batches ? (double)next / (double)stats.batches : 0;
  if (!lat_all.empty()) {
    std::vector<double> srt = lat_all;
    std::sort(srt.begin(), srt.end());
    auto pct = [&](double p) { return srt[std::min(srt.size() - 1, (size_t)(p * (double)(srt.size() - 1) + 0.5))]; };
    stats.p50_us = pct(0.50) * 1e6;
    stats.p99_us = pct(0.99) * 1e6;
  }
  stats.device_bytes = used;
  for (const ServeQueryResult& r : out) {
    stats.queries_admitted += r.admitted ? 1 : 0;
    for (const csm_result& x : r.results) {
      stats.results++;
      if (x.status == CSM_ST_CAPPED || x.status == CSM_ST_TIMED_OUT) stats.incomplete++;
    }
  }
  // attached queries go before their owner
  for (Ctx& a : att) if (a.h) { csm_gpu_destroy(a.h); a.h = nullptr; }
  return CSM_OK;
}

}  // namespace csm
