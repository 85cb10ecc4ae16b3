#!/usr/bin/env python3
"""Throughput benchmark of the continuous-subgraph-matching hot path.

Workload (default): the 2^22-vertex RMAT graph (average degree 28, 16 vertex
labels Zipf(1.2), 4 edge labels) with a 16-vertex dense query (>= 32 edges)
and an 80/20 insert/delete edge stream, per-update cap 10^6 matches (the
reference's --max-results), run by the SymBi plugin.  A step is one batch of
65,536 stream updates.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is batched updates/s with the stream
already in HBM (CUDA events on the engine's stream); `e2e` is the same metric
through the C ABI with pinned host buffers, the host->device copy of each
step's updates and the device->host read of its results inside the timed
region.  The plain one-update-per-launch form is measured on a sample of the
same stream from the same initial graph and must give identical counts.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "updates/s, p50/p99 update latency: batched vs plain GPU, bit-exact counts"
# DRAM bytes (read + write) of one search launch over a 16,384-update C3
# batch, from an ncu capture of that launch (dram__bytes_read.sum +
# dram__bytes_write.sum); scaled to a launch by the updates it processes.
SEARCH_DRAM_BYTES_PER_16384 = 50.7e9

CONFIGS = {
    "c3": {
        "preset": "c3", "algo": "parallel_symbi", "batch": 65536, "max_results": 1_000_000,
        "min_updates": 1_000_000,
        "workload": "RMAT 2^22 V, avg deg 28 (58.7M edges), 16 vlabels Zipf(1.2), 4 elabels; 16-vertex dense "
                    "query (avg deg >= 4); edge stream 80% insert / 20% delete; max_results 1e6 per update",
    },
    "c2": {
        "preset": "c2", "algo": "parallel_turboflux", "batch": 65536, "max_results": 1_000_000,
        "min_updates": 100_000,
        "workload": "RMAT 2^19 V, avg deg 16, 8 vlabels Zipf(1.0), 2 elabels; 8-vertex sparse query; "
                    "edge stream 90% insert / 10% delete; max_results 1e6 per update",
    },
    "c4": {
        "preset": "c4", "algo": "parallel_symbi", "batch": 65536, "max_results": 10_000,
        "min_updates": 200_000, "deadline_ms": 100,
        "workload": "C3 graph (RMAT 2^22 V, avg deg 28, 16 vlabels Zipf(1.2), 4 elabels); 64 standing queries of "
                    "4-32 vertices, half sparse, half dense, round-robin over SymBi / TurboFlux / GraphFlow; "
                    "Poisson edge stream 85% insert / 15% delete; 40 GB device-memory budget; per update max_results 1e4 "
                    "and a 100 ms search limit",
    },
    "c5": {
        "preset": "c5", "algo": "parallel_symbi", "batch": 8192, "max_results": 1_000_000,
        "min_updates": 500_000, "deadline_ns": 1_000_000_000,
        "workload": "RMAT 2^24 V, avg deg 32 (268M edges), 32 vlabels Zipf(1.0), 4 elabels; 24- and 32-vertex "
                    "queries (sparse and dense) as four standing queries on one graph, the CaLiG-style plugin on the "
                    "24-vertex sparse and 32-vertex dense ones, the NewSP-style plugin on the other two; 90/10 "
                    "insert/delete stream; per update max_results 1e6 and a 1 s limit",
    },
    "c1": {
        "preset": "c1", "algo": "parallel_graphflow", "batch": 2000, "max_results": 0, "min_updates": 2000,
        "workload": "RMAT 2^14 V, avg deg 8, 4 vlabels, 1 elabel; 6-vertex induced query; 2,000 insertions",
    },
}

CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={CLOCK_QUERY}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.device)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self) -> dict:
        self.f.flush()
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def cuda_view(ptr: int, nbytes: int, device: int):
    """torch uint8 view of raw device memory (no copy)."""
    import torch

    class _Arr:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}
    return torch.as_tensor(_Arr(), device=f"cuda:{device}")


def stream_plan(cfg: dict, warmup: int, steps: int, e2e_steps: int = 2) -> tuple[int, int]:
    """(stream length, first timed update): the same for the GPU arm and the reference arm, so
    both generate one workload and time the same updates.  The first `warmup` batches are the
    warm-up; the timed window starts at update warmup * batch."""
    B = cfg["batch"]
    return max(cfg["min_updates"], (warmup + max(steps, e2e_steps)) * B), warmup * B


def bench_config(cfg: dict, args, world: int) -> dict:
    """The `config` object of both arms' JSON lines (built by one function so that they match)."""
    n_updates, first = stream_plan(cfg, args.warmup, args.steps, args.e2e_steps)
    return {"workload": cfg["workload"], "plugin": cfg["algo"], "batch": cfg["batch"], "stream_updates": n_updates,
            "first_timed_update": first, "updates_timed": args.steps * cfg["batch"],
            "max_results": cfg["max_results"],
            "tail": "enumerated" if args.tail_enumerate else "counted (independent tail of each order)",
            "l2": "inputs larger than L2 (graph ~3.4 GB in HBM)",
            "parallelism": f"seed-sharded x{world} (replicated graph, one all-reduce per batch)"
            if world > 1 else "single GPU"}


def get_workload(cfg: dict, n_updates: int, snapshot_at: int = 0):
    """Seeded workload; with snapshot_at the generator also writes the data graph as it stands
    after the first snapshot_at updates (data_at_<n>.bin), where runs of the reference start."""
    from paracosm_b200 import workload
    base = Path(os.environ.get("CSM_BENCH_DIR", "/tmp/csm_bench"))
    d = base / f"{cfg['preset']}_{n_updates}"
    t0 = time.perf_counter()
    extra = ["--snapshot-at", str(snapshot_at)] if snapshot_at else None
    w = workload.generate(cfg["preset"], d, updates=n_updates, extra=extra)
    log(f"workload {d} ready in {time.perf_counter() - t0:.1f}s: {len(w.vlabels)} V, {len(w.edges)} E, "
        f"{len(w.stream)} updates")
    return w


class RefRun:
    """One run of the reference compiled from its sources (oracle/_ref/ref_driver: the unmodified
    plugin objects driven in the sequential update order) over the stream from update `first`,
    starting from the data graph as it stands there.  Gated runs load and preprocess at once
    and start their timed update loop only when `go()` is called, so that timed loops never
    overlap.  A watchdog ends a run `budget` seconds into its update loop, even inside an update
    (parallel TurboFlux ignores the result cap below depth 2)."""

    def __init__(self, w, algo: str, threads: int, cap: int, first: int, budget: float, gated: bool, tag: str,
                 apply: bool = False):
        """apply: start from the initial graph and let the reference's Graph apply the first `first`
        updates itself (--apply-to) instead of loading the generator's snapshot there."""
        self.algo, self.threads, self.first, self.budget = algo, threads, first, budget
        self.tmp = Path(tempfile.mkdtemp(prefix=f"csm_ref_{tag}_"))
        self.out = self.tmp / "rows.csv"
        self.gate = self.tmp / "gate" if gated else None
        self.proc = None
        self.err = None
        drv = ROOT / "oracle" / "_ref" / "ref_driver"
        if not drv.exists():
            self.err = "reference driver not built (oracle/_ref/ref_driver)"
            return
        graph = w.directory / (f"data_at_{first}.bin" if first and not apply else "data.bin")
        start = ["--apply-to", str(first)] if apply and first else ["--first", str(first)]
        cmd = [str(drv), "-q", str(w.query_path(0)), "-D", str(graph), "-U", str(w.directory / "stream.bin"),
               "-a", algo, "-t", str(threads)] + start + ["--wall-budget", str(budget), "--out", str(self.out)]
        if cap:
            cmd += ["--max-results", str(cap)]
        if gated:
            cmd += ["--gate", str(self.gate)]
        self.t0 = time.perf_counter()
        self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)

    def wait_ready(self, timeout: float) -> bool:
        if self.proc is None or self.gate is None:
            return False
        ready = Path(str(self.gate) + ".ready")
        t0 = time.perf_counter()
        while not ready.exists():
            if self.proc.poll() is not None:
                self.err = f"reference driver exited ({self.proc.returncode}) before its updates: " + \
                    self.proc.stderr.read()[-300:]
                return False
            if time.perf_counter() - t0 > timeout:
                self.err = f"reference driver not ready within {timeout:.0f}s"
                return False
            time.sleep(0.2)
        return True

    def go(self) -> None:
        Path(str(self.gate) + ".go").touch()

    def collect(self, hard_timeout: float) -> dict | None:
        """updates/s = updates completed / seconds of the update loop, plus latency percentiles."""
        if self.proc is None:
            return None
        try:
            stdout, stderr = self.proc.communicate(timeout=hard_timeout)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            self.proc.communicate()
            self.err = f"reference driver did not finish within {hard_timeout:.0f}s"
            return None
        done, elapsed, note = None, None, ""
        for line in stdout.splitlines():
            if "updates_done=" in line:
                kv = dict(x.split("=", 1) for x in line.split() if "=" in x)
                done, elapsed = int(kv["updates_done"]), float(kv["elapsed_s"])
                if line.startswith("wall_budget_reached"):
                    note = "(budget reached inside an update)"
        if done is None:
            self.err = f"reference driver failed (exit {self.proc.returncode}): {stderr[-300:]}"
            return None
        rows = self.rows()
        lat = rows["latency_ns"].astype(np.float64) if len(rows) else np.zeros(0)
        if done == 0 or elapsed <= 0:
            self.err = f"no update finished within {self.budget:.0f}s {note}".strip()
            return None
        return {"updates": int(done), "seconds": elapsed, "value": done / elapsed,
                "first_update": self.first, "last_update": self.first + int(done) - 1,
                "p50_us": float(np.percentile(lat, 50)) / 1e3 if len(lat) else None,
                "p99_us": float(np.percentile(lat, 99)) / 1e3 if len(lat) else None,
                "wall_s": time.perf_counter() - self.t0, "note": note, "algo": self.algo, "threads": self.threads}

    def rows(self) -> np.ndarray:
        """Per-update rows written so far (stream index, pos, neg, latency)."""
        dt = np.dtype([("idx", "<i8"), ("pos", "<u8"), ("neg", "<u8"), ("latency_ns", "<u8")])
        if not self.out.exists():
            return np.zeros(0, dtype=dt)
        vals = []
        for line in self.out.read_text().splitlines()[1:]:
            parts = line.split(",")
            if len(parts) >= 10:
                vals.append((int(parts[0]), int(parts[6]), int(parts[7]), int(parts[8])))
        return np.array(vals, dtype=dt)

    def kill(self) -> None:
        if self.proc is not None and self.proc.poll() is None:
            self.proc.kill()
            self.proc.communicate()


def cpu_line(r: RefRun, res: dict | None, cfg) -> dict:
    if res is None:
        return {"value": None, "unit": "updates/s", "cores": r.threads, "kind": "reference", "sample": r.err}
    return {"value": res["value"], "unit": "updates/s", "cores": res["threads"], "kind": "reference",
            "updates": res["updates"], "first_update": res["first_update"], "last_update": res["last_update"],
            "sample": f"stream updates {res['first_update']}..{res['last_update']} ({res['updates']} updates) in "
                      f"{res['seconds']:.1f}s of incremental matching from the data graph as it stands at update "
                      f"{res['first_update']}, {res['algo']} -t {res['threads']} (reference sources, sequential "
                      f"update order, max_results {cfg['max_results']}), {r.budget:.0f}s budget {res['note']}".strip(),
            "p50_us": res["p50_us"], "p99_us": res["p99_us"]}


def start_timed_refs(w, cfg, first: int, budget: float) -> list[RefRun]:
    """The reference on the host cores from the first timed update: parallel_turboflux on every
    core (the baseline the targets are stated against), then sequential SymBi on one core, which
    stops at exactly max_results as the engine does.  Both load at once; their timed loops run
    one after the other (run_timed_refs)."""
    ncpu = os.cpu_count() or 2
    return [RefRun(w, "parallel_turboflux", ncpu, cfg["max_results"], first, budget, True, "tf"),
            RefRun(w, "symbi", 1, cfg["max_results"], first, budget, True, "sy")]


def run_timed_refs(refs: list[RefRun], cfg, budget: float) -> list[dict]:
    out = []
    for r in refs:
        res = None
        if r.wait_ready(3600):
            r.go()
            res = r.collect(budget + 600)
        else:
            r.kill()
        out.append(cpu_line(r, res, cfg))
    return out


def start_parity_refs(w, cfg, end: int, budget: float) -> list[RefRun]:
    """Sequential SymBi (the reference plugin that stops at exactly max_results, as the engine does)
    on several segments of the stream [0, end) at once, each starting where its segment begins
    (the reference's Graph applies the earlier updates itself): one run gets stuck on the rare
    update whose search takes minutes, the others keep comparing.  As many runs as host cores
    and memory allow (a run holds about 9 GB at 2^22 vertices), at most 12."""
    try:
        import psutil
        mem_gb = psutil.virtual_memory().available / 2**30
    except Exception:
        mem_gb = 64.0
    n = int(max(1, min(12, (os.cpu_count() or 2) - 2, (mem_gb - 40) // 10)))
    return [RefRun(w, "symbi", 1, cfg["max_results"], (k * end // n) // 1000 * 1000, budget, True, f"par{k}",
                   apply=True) for k in range(n)]


def parity_check(rows: np.ndarray, gpu: np.ndarray, base: int, cap: int) -> dict:
    """Per-update pos / neg / capped of the engine (gpu[i] is stream update base + i) against the
    reference's rows; a reference count at the cap is a capped update (it stops at exactly the cap)."""
    sel = rows[(rows["idx"] >= base) & (rows["idx"] < base + len(gpu))]
    if len(sel) == 0:
        return {"updates_compared": 0, "mismatches": 0}
    g = gpu[sel["idx"] - base]
    ref_capped = (sel["pos"] + sel["neg"] >= cap) if cap else np.zeros(len(sel), bool)
    bad = (g["pos"] != sel["pos"]) | (g["neg"] != sel["neg"]) | ((g["status"] == 1) != ref_capped) | \
        (g["status"] >= 2)
    out = {"updates_compared": int(len(sel)), "mismatches": int(bad.sum()), "first_update": int(sel["idx"][0]),
           "last_update": int(sel["idx"][-1]), "nonzero_updates": int(((sel["pos"] + sel["neg"]) > 0).sum()),
           "matches": int(sel["pos"].sum() + sel["neg"].sum()), "capped": int(ref_capped.sum())}
    if bad.any():
        k = int(np.nonzero(bad)[0][0])
        out["first_mismatch"] = {"update": int(sel["idx"][k]), "ref": [int(sel["pos"][k]), int(sel["neg"][k])],
                                 "gpu": [int(g["pos"][k]), int(g["neg"][k]), int(g["status"][k])]}
    return out


def run_reference_arm(args, cfg):
    """The reference's CPU implementation on this host, on the same workload, config and update
    range as the GPU arm: parallel_turboflux on every core (value) and sequential SymBi on one
    core beside it, both from the data graph at the GPU arm's first timed update."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    n_updates, first = stream_plan(cfg, args.warmup, args.steps, args.e2e_steps)
    w = get_workload(cfg, n_updates, snapshot_at=first)
    budget = float(os.environ.get("CSM_REF_BUDGET_S", "60"))
    tf, sy = run_timed_refs(start_timed_refs(w, cfg, first, budget), cfg, budget)
    line = {"impl": "reference", "metric": METRIC, "unit": "updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "dtype": "u32", "data": "synthetic", "config": bench_config(cfg, args, world)}
    if tf["value"] is None:
        line.update({"value": None, "unavailable": tf["sample"]})
    else:
        line.update({"value": tf["value"], "ms_per_step": 1000.0 / tf["value"], "p50_us": tf.get("p50_us"),
                     "p99_us": tf.get("p99_us"), "cpu_baseline": tf,
                     "e2e": {"value": tf["value"], "unit": "updates/s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0}})
    line["sequential_symbi_capped"] = sy
    print(json.dumps(line), flush=True)


def serve_sweep(w, cfg, rates, seconds, *, n_queries, device=0, plugins=None, cap=None,
                deadline_ms=None) -> list[dict]:
    """Runs the serving loop (paracosm_b200/_bin/csm_serve) on the workload: one process, one set-up,
    then `seconds` of Poisson arrivals at each offered rate in turn (each segment continues the
    stream where the last one stopped).  One dict per rate."""
    exe = ROOT / "paracosm_b200" / "_bin" / "csm_serve"
    cmd = [str(exe), "-w", str(w.directory), "--queries", str(n_queries), "--rates", ",".join(f"{r:g}" for r in rates),
           "--max-seconds", str(seconds), "--max-batch", str(cfg["batch"]), "--device", str(device),
           "--cap", str(cfg["max_results"] if cap is None else cap),
           "--plugins", ",".join(plugins or [cfg["algo"]]), "--graphs", "1"]
    if deadline_ms:
        cmd += ["--deadline-ms", str(deadline_ms)]
    t0 = time.perf_counter()
    limit = 600.0 + 60.0 * seconds * len(rates)
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=limit)
    except subprocess.TimeoutExpired:
        return [{"offered_rate": r, "error": f"serving run exceeded {limit:.0f}s"} for r in rates]
    if p.returncode != 0:
        return [{"offered_rate": r, "error": p.stderr[-300:]} for r in rates]
    out = [json.loads(line) for line in p.stdout.strip().splitlines() if line.startswith('{"segment"')]
    wall = time.perf_counter() - t0
    for d in out:
        d["process_wall_s"] = wall
        log(f"serve rate {d['offered_rate']:g}: sustained {d['sustained']:.0f} upd/s p50 {d['p50_us']:.0f} us "
            f"p99 {d['p99_us']:.0f} us mean batch {d['mean_batch']:.0f}")
    return out


C4_PLUGINS = ["parallel_symbi", "parallel_turboflux", "parallel_graphflow"]
C5_PLUGINS = ["parallel_calig", "parallel_newsp", "parallel_newsp", "parallel_calig"]


def c4_leg(rates, seconds, device=0) -> dict:
    """C4: 64 standing queries (sizes 4-32, half sparse, half dense, round-robin over the three
    plugins) on the 2^22-vertex graph, Poisson arrivals swept over the offered rates, admission
    against a 40 GB budget, with the per-update cap and search limit named in the config."""
    cfg = CONFIGS["c4"]
    w = get_workload(cfg, cfg["min_updates"])
    sweep = serve_sweep(w, cfg, rates, seconds, n_queries=64, plugins=C4_PLUGINS,
                        deadline_ms=cfg.get("deadline_ms"), device=device)
    ok = [d for d in sweep if "sustained" in d]
    best = max(ok, key=lambda d: d["sustained"]) if ok else None
    return {"workload": cfg["workload"], "queries": 64, "plugins": C4_PLUGINS, "max_results": cfg["max_results"],
            "deadline_ms": cfg["deadline_ms"], "budget_gb": 40, "seconds_per_rate": seconds,
            "sustained_best": best["sustained"] if best else None,
            "p50_us_at_best": best["p50_us"] if best else None, "p99_us_at_best": best["p99_us"] if best else None,
            "sweep": sweep,
            "note": "max_results 1e4 and a 100 ms search limit per update are not in the config's text: with the "
                    "1e6 cap of the 2^22-vertex SymBi config, 32-vertex sparse queries reach the cap on most "
                    "updates and a first batch does not finish"}


def run_serving_config(args, cfg):
    """C4 on its own: value = the highest sustained updates/s of the sweep."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    rates = [float(r) for r in (args.serve_rates or "1e4,1e5,1e6").split(",") if r]
    leg = c4_leg(rates, args.serve_seconds)
    line = {"metric": METRIC, "value": leg["sustained_best"], "unit": "updates/s", "n_gpus": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "batch": cfg["batch"], "max_results": cfg["max_results"]},
            "p50_us": leg["p50_us_at_best"], "p99_us": leg["p99_us_at_best"], "serving": leg["sweep"], "c4": leg}
    print(json.dumps(line), flush=True)


def c5_leg(warmup: int, steps: int, device=0) -> dict:
    """C5: the four large queries (24 and 32 vertices, sparse and dense) as standing queries on one
    2^24-vertex graph, run by the CaLiG-style and NewSP-style plugins (each takes one sparse and one
    dense query), batches of 8,192 updates, per update a cap of 1e6 matches and a 1 s limit.
    updates/s from CUDA events on the owner's stream (the attached queries' streams join it);
    success rate = share of (update, query) results neither CAPPED nor TIMED_OUT."""
    import torch

    from paracosm_b200 import ST_CAPPED, ST_TIMED_OUT, Engine
    cfg = CONFIGS["c5"]
    B, W, K = cfg["batch"], warmup, steps
    w = get_workload(cfg, max(cfg["min_updates"], (W + K) * B))
    plugins = C5_PLUGINS
    t0 = time.perf_counter()
    own = Engine(plugins[0], max_results=cfg["max_results"], max_batch=B, deadline_ns=cfg["deadline_ns"],
                 graphs=True, device=device)
    qv0, qe0 = w.queries[0]
    own.set_query(qv0, qe0)
    vls = np.concatenate([q[0] for q in w.queries])
    els = np.concatenate([q[1][:, 2] for q in w.queries])
    own.reserve_labels(np.unique(vls), np.unique(els))
    own.load_graph(w.vlabels, w.edges)
    own.build_index()
    att = [own.attach(*w.queries[i], plugins[i % len(plugins)], max_results=cfg["max_results"])
           for i in range(1, len(w.queries))]
    log(f"C5 engine with {len(w.queries)} queries ready in {time.perf_counter() - t0:.1f}s")
    for i in range(W):
        own.run(w.stream[i * B:(i + 1) * B])
    ext = torch.cuda.ExternalStream(own.stream(), device=f"cuda:{device}")
    res = [[] for _ in range(len(w.queries))]
    ms = 0.0
    for k in range(K):
        chunk = np.ascontiguousarray(w.stream[(W + k) * B:(W + k + 1) * B])
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(ext)
        first = own.submit(chunk)
        b.record(ext)
        b.synchronize()
        ms += a.elapsed_time(b)
        own.wait()
        res[0].append(own.results(first, len(chunk)))
        for i, q in enumerate(att):
            res[i + 1].append(q.results(first, len(chunk)))
    per_q = []
    for i, rs in enumerate(res):
        r = np.concatenate(rs)
        bad = (r["status"] == ST_CAPPED) | (r["status"] == ST_TIMED_OUT)
        per_q.append({"query": i, "vertices": int(len(w.queries[i][0])), "edges": int(len(w.queries[i][1])),
                      "plugin": plugins[i % len(plugins)], "success_rate": float(1 - bad.mean()),
                      "capped": int((r["status"] == ST_CAPPED).sum()),
                      "timed_out": int((r["status"] == ST_TIMED_OUT).sum()),
                      "p50_us": float(np.percentile(r["latency_ns"], 50)) / 1e3,
                      "p99_us": float(np.percentile(r["latency_ns"], 99)) / 1e3})
    allr = np.concatenate([np.concatenate(rs) for rs in res])
    bad = (allr["status"] == ST_CAPPED) | (allr["status"] == ST_TIMED_OUT)
    for q in att:
        q.close()
    own.close()
    return {"workload": cfg["workload"], "batch": B, "warmup_batches": W, "timed_batches": K,
            "max_results": cfg["max_results"], "deadline_ns": cfg["deadline_ns"],
            "updates_per_s": K * B / (ms / 1e3) if ms > 0 else None, "ms_per_batch": ms / K if K else None,
            "success_rate": float(1 - bad.mean()), "queries": per_q,
            "timing": "CUDA events on the owner's stream around each submit (all four queries' searches)"}


def run_stress_config(args, cfg):
    """C5 on its own: value = updates/s over the timed batches."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    leg = c5_leg(args.warmup, args.steps)
    line = {"metric": METRIC, "value": leg["updates_per_s"], "unit": "updates/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": leg["ms_per_batch"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "batch": cfg["batch"], "max_results": cfg["max_results"],
                       "deadline_ns": cfg["deadline_ns"]},
            "success_rate": leg["success_rate"], "c5": leg}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c3")
    ap.add_argument("--algo", default=None)
    ap.add_argument("--batch", type=int, default=None)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--plain-sample", type=int, default=3000)
    ap.add_argument("--cpu-budget", type=float, default=30.0,
                    help="seconds of update loop for each timed reference run")
    ap.add_argument("--parity-budget", type=float, default=45.0,
                    help="seconds of update loop for the reference SymBi run the counts are checked against")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the search-shape autotuner")
    ap.add_argument("--tail-enumerate", action="store_true",
                    help="enumerate the independent tail of each order instead of counting it")
    ap.add_argument("--serve-rates", default="1e4,1e5,1e6",
                    help="offered loads (updates/s) for the serving-loop leg; empty to skip")
    ap.add_argument("--serve-seconds", type=float, default=4.0)
    ap.add_argument("--extra-configs", default="c4,c5",
                    help="bounded legs of the other configs added to the default line (c4: 64 standing queries "
                         "served over a rate sweep; c5: large queries with the CaLiG- and NewSP-style plugins); "
                         "empty to skip")
    ap.add_argument("--c4-seconds", type=float, default=8.0, help="seconds of arrivals per offered rate (C4 leg)")
    args = ap.parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.algo:
        cfg["algo"] = args.algo
    if args.batch:
        cfg["batch"] = args.batch
    if args.impl == "reference":
        return run_reference_arm(args, cfg)
    if args.config == "c4":
        return run_serving_config(args, cfg)
    if args.config == "c5":
        return run_stress_config(args, cfg)

    import torch
    import torch.distributed as dist

    from paracosm_b200 import RESULT_DTYPE, Engine, workload
    from paracosm_b200.shard import allreduce_results

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = local
    B, W, K, KE = cfg["batch"], args.warmup, args.steps, args.e2e_steps
    n_updates, first = stream_plan(cfg, W, K, KE)
    w = get_workload(cfg, n_updates, snapshot_at=first)
    qv, qe = w.queries[0]
    stream = w.stream
    assert len(stream) >= (W + max(K, KE)) * B

    # ---- the reference on the host cores (rank 0, one GPU): the timed runs load now and
    # start their update loops after the GPU legs; the parity run (sequential SymBi from the
    # initial graph, the warm-up batches' updates) runs meanwhile ----
    cpu_refs, par_refs = [], []
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu_refs = start_timed_refs(w, cfg, first, args.cpu_budget)
        par_refs = start_parity_refs(w, cfg, (W + K) * B, args.parity_budget)

    # ---- batched engine, inputs resident in HBM ----
    t0 = time.perf_counter()
    # N > 1: every rank holds a replica and applies every batch; root tasks are dealt
    # across ranks and one all-reduce per batch combines the per-update results
    te = bool(args.tail_enumerate)
    eng = Engine(cfg["algo"], max_results=cfg["max_results"], max_batch=B, device=dev,
                 shard_rank=rank if world > 1 else 0, shard_count=world, tail_enumerate=te)
    eng.set_query(qv, qe)
    eng.load_graph(w.vlabels, w.edges)
    eng.build_index()
    log(f"engine ready in {time.perf_counter() - t0:.1f}s")
    shape = None
    if not args.no_tune:
        t1 = time.perf_counter()
        shape = eng.autotune(np.ascontiguousarray(stream[:B]))
        log(f"autotuned search shape {shape} in {time.perf_counter() - t1:.1f}s")
    d_stream = torch.from_numpy(stream[: (W + K) * B].view(np.uint8).copy()).to(f"cuda:{dev}")
    ext = torch.cuda.ExternalStream(eng.stream(), device=f"cuda:{dev}")
    res_dev = torch.empty(K * B * RESULT_DTYPE.itemsize, dtype=torch.uint8, device=f"cuda:{dev}")
    warm_res = []
    for i in range(W):
        f0 = eng.submit_device(d_stream.data_ptr() + i * B * 16, B)
        eng.wait()
        warm_res.append(eng.results(f0, B))
    warm_res = np.concatenate(warm_res) if warm_res else np.zeros(0, dtype=RESULT_DTYPE)
    if world > 1:
        t = torch.from_numpy(warm_res.view(np.int64).reshape(-1, 6).copy()).to(f"cuda:{dev}")
        allreduce_results(t, cap=cfg["max_results"])
        warm_res = t.cpu().numpy().view(RESULT_DTYPE).reshape(-1)
    st0 = eng.stats()
    launches0 = eng.kernel_launches()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
    with ClockSampler(dev) as clk:
        evs[0].record(ext)
        for k in range(K):
            eng.submit_device(d_stream.data_ptr() + (W + k) * B * 16, B)
            rp, rn = eng.results_device()
            with torch.cuda.stream(ext):
                view = cuda_view(rp, rn * RESULT_DTYPE.itemsize, dev)
                if world > 1:
                    allreduce_results(view.view(torch.int64).view(-1, 6), cap=cfg["max_results"])
                res_dev[k * B * RESULT_DTYPE.itemsize:(k + 1) * B * RESULT_DTYPE.itemsize].copy_(view)
            evs[k + 1].record(ext)
        evs[K].synchronize()
        eng.wait()
    torch.cuda.synchronize()
    ms = evs[0].elapsed_time(evs[K])
    batch_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(K)]
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    st1 = eng.stats()
    launches = eng.kernel_launches() - launches0
    res = np.frombuffer(res_dev.cpu().numpy().tobytes(), dtype=RESULT_DTYPE)
    value = K * B / (ms / 1e3)  # each update counted once, whatever the number of ranks
    lat = res["latency_ns"].astype(np.float64)
    search_ms = st1["search_ms"] - st0["search_ms"]
    search_n = st1["search_launches"] - st0["search_launches"]
    work = float(res["work_bytes"].sum())
    peak, peak_kind = measured_peak_hbm()
    achieved = (work / 1e9) / (search_ms / 1e3) if search_ms > 0 else 0.0

    eng.close()

    # ---- e2e through the C ABI with pinned host buffers: a second engine from the
    # same initial graph replays the warm-up batches, then takes the first KE timed
    # batches of the stream from host memory (the same updates as the device-resident
    # timed region starts with) ----
    kw = {k: shape[k] for k in ("warps_per_block", "blocks_per_sm", "donate_every", "split_deep")} if shape else {}
    eng = Engine(cfg["algo"], max_results=cfg["max_results"], max_batch=B, device=dev,
                 shard_rank=rank if world > 1 else 0, shard_count=world, tail_enumerate=te, **kw)
    eng.set_query(qv, qe)
    eng.load_graph(w.vlabels, w.edges)
    eng.build_index()
    ext = torch.cuda.ExternalStream(eng.stream(), device=f"cuda:{dev}")
    for i in range(W):
        eng.submit_device(d_stream.data_ptr() + i * B * 16, B)
        eng.wait()
    host = torch.from_numpy(stream[W * B:(W + KE) * B].view(np.uint8).copy()).pin_memory()
    e2e_ms = 0.0
    e2e_same = True
    for k in range(KE):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(ext)
        f0 = eng.submit_ptr(host.data_ptr() + k * B * 16, B)
        r = eng.results(f0, B)
        if world > 1:
            t = torch.from_numpy(r.view(np.int64).reshape(-1, 6).copy()).to(f"cuda:{dev}")
            allreduce_results(t, cap=cfg["max_results"])
            r = t.cpu().numpy().view(RESULT_DTYPE).reshape(-1)
        b.record(ext)
        b.synchronize()
        e2e_ms += a.elapsed_time(b)
        assert len(r) == B
        if k < K:
            seg = res[k * B:(k + 1) * B]
            e2e_same &= bool(np.array_equal(r["pos"], seg["pos"]) and np.array_equal(r["neg"], seg["neg"]))
    if world > 1:
        t = torch.tensor([e2e_ms], device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = KE * B / (e2e_ms / 1e3) if e2e_ms > 0 else None
    eng.close()

    # ---- plain form (one update per launch sequence) on the first updates of the timed
    # window, from the data graph as it stands there: the same updates, in the same graph
    # state, as the batched form's first timed batch and the reference runs ----
    plain = None
    if rank == 0 and args.plain_sample > 0:
        P = min(args.plain_sample, K * B)
        sample = np.ascontiguousarray(stream[first:first + P])
        svl, sedges = workload.read_graph(w.directory / f"data_at_{first}.bin")
        forms = {}
        for graphs in (False,):
            peng = Engine(cfg["algo"], max_results=cfg["max_results"], mode="plain", device=dev, graphs=graphs,
                          tail_enumerate=te, **kw)
            peng.set_query(qv, qe)
            peng.load_graph(svl, sedges)
            peng.build_index()
            torch.cuda.synchronize()
            l0 = peng.kernel_launches()
            t1 = time.perf_counter()
            pr = peng.run(sample)
            plain_s = time.perf_counter() - t1
            pst = peng.stats()
            same = bool(np.array_equal(pr["pos"], res["pos"][:P]) and np.array_equal(pr["neg"], res["neg"][:P]) and
                        np.array_equal(pr["status"], res["status"][:P]))
            # one submit of P updates, one launch sequence each: an update's service time is the gap
            # between its completion stamp and the previous one's
            svc = np.diff(np.concatenate([[0], np.sort(pr["latency_ns"].astype(np.float64))]))
            # launches per update: the label-triple test decides the sequence (2-3 launches when no
            # query edge matches, about 9 otherwise); reported as the mean and per class
            lpu = np.array(peng.kernel_launches() - l0, dtype=np.float64) / P
            forms[graphs] = {"value": P / plain_s, "updates": P, "first_update": first, "device_ms": pst["total_device_ms"],
                             "p50_us": float(np.percentile(svc, 50)) / 1e3,
                             "p99_us": float(np.percentile(svc, 99)) / 1e3,
                             "kernel_launches_per_update": float(lpu),
                             "counts_equal_batched": same}
            peng.close()
        plain = dict(forms[False], form="one update per launch sequence, launched from the host")

    # ---- serving loop: Poisson arrivals admitted in continuous batches ----
    serving = None
    if rank == 0 and world == 1 and args.serve_rates:
        serving = serve_sweep(w, cfg, [float(r) for r in args.serve_rates.split(",") if r], args.serve_seconds,
                              n_queries=1, device=dev)

    # ---- the reference: parity of the counts, then the timed runs one after another ----
    cpu, cpu_seq, parity, checks = None, None, None, {}
    if par_refs:
        # the engine's results for updates [0, (W + K) * B): warm-up batches, then the timed window
        gpu_all = np.concatenate([warm_res, res])
        for r in par_refs:
            if r.wait_ready(3600):
                r.go()
        for k, r in enumerate(par_refs):
            r.collect(args.parity_budget + 600)
            checks[f"segment_{k}"] = parity_check(r.rows(), gpu_all, 0, cfg["max_results"])
        parity = {"reference": "symbi -t 1 (reference sources, sequential update order, cap-honouring), "
                               f"{len(par_refs)} runs on segments of the stream, {args.parity_budget:.0f}s each",
                  "engine": "batched: the warm-up batches and the timed window"}
    if cpu_refs:
        cpu, cpu_seq = run_timed_refs(cpu_refs, cfg, args.cpu_budget)
        # the sequential SymBi run times the first updates of the timed window: its counts too
        checks["timed_window"] = parity_check(cpu_refs[1].rows(), res, first, cfg["max_results"])
    if parity is not None:
        parity.update(checks)
        parity["updates_compared"] = sum(c["updates_compared"] for c in checks.values())
        parity["mismatches"] = sum(c["mismatches"] for c in checks.values())
        log(f"parity against the reference SymBi: {parity['updates_compared']} updates, "
            f"{parity['mismatches']} mismatches")

    # ---- bounded legs of the serving (C4) and large-query (C5) configs ----
    extra = {}
    extras = [x for x in args.extra_configs.split(",") if x] if (rank == 0 and world == 1) else []
    if "c4" in extras:
        t1 = time.perf_counter()
        extra["c4"] = c4_leg([1e4, 1e5, 1e6], args.c4_seconds, device=dev)
        extra["c4"]["wall_s"] = time.perf_counter() - t1
    if "c5" in extras:
        t1 = time.perf_counter()
        extra["c5"] = c5_leg(1, 2, device=dev)
        extra["c5"]["wall_s"] = time.perf_counter() - t1

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None,
            "dtype": "u32", "data": "synthetic",
            "config": bench_config(cfg, args, world),
            "search_shape": shape,
            "timed_window": {"first_update": first, "last_update": first + K * B - 1, "per_batch_ms": batch_ms},
            "p50_us": float(np.percentile(lat, 50)) / 1e3, "p99_us": float(np.percentile(lat, 99)) / 1e3,
            "plain": plain,
            "batched_over_plain": (value / plain["value"]) if plain else None,
            "serving": serving,
            "e2e": {"value": e2e_value, "unit": "updates/s", "h2d_bytes_per_step": B * 16,
                    "d2h_bytes_per_step": B * RESULT_DTYPE.itemsize, "first_update": first,
                    "counts_equal_device_resident": e2e_same},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if peak else None,
                         "traffic": SEARCH_DRAM_BYTES_PER_16384 * B / 16384 if cfg["preset"] == "c3" else None,
                         "traffic_note": "ncu dram__bytes_read+write of a 16384-update C3 launch, scaled by updates",
                         "peak_kind": peak_kind, "kernel": "k_search", "launches": search_n,
                         "kernel_ms": search_ms, "algorithmic_bytes": work},
            "cpu_baseline": cpu,
            "cpu_baseline_sequential_symbi_capped": cpu_seq,
            "parity": parity,
            **extra,
            "gpu_launches": launches,
            "clocks": clocks,
            "counts": {"positive": int(res["pos"].sum()), "negative": int(res["neg"].sum()),
                       "capped": int((res["status"] == 1).sum()), "invalid": int((res["status"] == 3).sum()),
                       "unsafe": int(((res["pos"] + res["neg"]) > 0).sum())},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
