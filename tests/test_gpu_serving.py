"""The serving loop (paracosm_b200/_bin/csm_serve): updates arrive as a Poisson
stream and are admitted in continuous batches whose sizes follow the arrivals;
standing queries arrive while updates are being served.  Every query's
per-update results equal the results of the same query run alone over the
same stream, whatever the batches were."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from paracosm_b200 import RESULT_DTYPE, Engine, workload

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
SERVE = ROOT / "paracosm_b200" / "_bin" / "csm_serve"
PLUGINS = ["parallel_symbi", "parallel_turboflux", "parallel_graphflow"]
QUERIES = ["6:sparse:1", "4:dense", "7:sparse:2", "5:dense", "9:sparse:1"]


@pytest.fixture(scope="module")
def wl(tmp_path_factory):
    extra = ["--log2-n", "13", "--avg-degree", "10", "--vlabels", "4", "--zipf", "0.8", "--elabels", "2",
             "--updates", "6000", "--insert-frac", "0.8"]
    for q in QUERIES:
        extra += ["--query", q]
    d = tmp_path_factory.mktemp("serve") / "w"
    return d, workload.generate("c2", d, extra=extra)


def read_results(path: Path) -> list[dict]:
    b = path.read_bytes()
    assert b[:4] == b"CSMR"
    nq = int(np.frombuffer(b, np.uint32, 1, 4)[0])
    off, out = 8, []
    for _ in range(nq):
        adm = int(np.frombuffer(b, np.uint32, 1, off)[0])
        first, cnt = (int(x) for x in np.frombuffer(b, np.uint64, 2, off + 4))
        off += 20
        res = np.frombuffer(b, RESULT_DTYPE, cnt, off).copy()
        off += cnt * RESULT_DTYPE.itemsize
        out.append({"admitted": bool(adm), "first": first, "res": res})
    return out


def alone(w, i, cap):
    qv, qe = w.queries[i]
    with Engine(PLUGINS[i % 3], max_results=cap, want_hash=True) as eng:
        eng.set_query(qv, qe)
        eng.load_graph(w.vlabels, w.edges)
        eng.build_index()
        return eng.run(w.stream)


def run_serve(d, tmp_path, *args):
    out = tmp_path / "res.bin"
    r = subprocess.run([str(SERVE), "-w", str(d), "--hash", "1", "--out", str(out), *args], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1]), read_results(out)


@pytest.mark.parametrize("graphs", ["0", "1"])
def test_results_alone_and_in_the_served_mix(wl, tmp_path, graphs):
    d, w = wl
    cap = 2000
    # 6000 updates at 40k/s: about 0.15 s of arrivals; the later queries
    # arrive while updates are being served
    summary, res = run_serve(d, tmp_path, "--rate", "40000", "--cap", str(cap), "--arrive-every", "0.03",
                             "--max-batch", "1024", "--graphs", graphs)
    assert summary["updates"] == len(w.stream)
    assert summary["batches"] > 1 and summary["mean_batch"] < len(w.stream)
    assert summary["queries_admitted"] == len(QUERIES)
    assert summary["p99_us"] >= summary["p50_us"] > 0
    late = 0
    for i, r in enumerate(res):
        assert r["admitted"]
        ref = alone(w, i, cap)[r["first"]:]
        got = r["res"]
        assert len(got) == len(ref)
        for k in ("pos", "neg", "status", "hash"):
            assert np.array_equal(got[k], ref[k]), (i, k, np.nonzero(got[k] != ref[k])[0][:10])
        late += r["first"] > 0
    assert late >= 1  # at least one query arrived mid-stream


def test_queries_beyond_the_budget_are_refused(wl, tmp_path):
    d, w = wl
    summary, res = run_serve(d, tmp_path, "--rate", "1e6", "--budget-gb", "0.000001", "--max-updates", "500")
    assert summary["queries_admitted"] == 1 and summary["queries_refused"] == len(QUERIES) - 1
    assert res[0]["admitted"] and not any(r["admitted"] for r in res[1:])
    assert len(res[0]["res"]) == 500
