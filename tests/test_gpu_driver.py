"""The csm driver on the GPU: its summary lines and per-update output equal the
reference's sequential counts (golden fixtures) and the InitialMatching count
the reference's own csm prints."""
from __future__ import annotations

import csv
import json
import subprocess

import numpy as np
import pytest

from conftest import load_golden
from test_driver import CSM

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["batched", "plain"])
@pytest.mark.parametrize("algo", ["parallel_graphflow", "parallel_turboflux", "parallel_symbi"])
def test_driver_output_matches_the_reference(tmp_path, algo, mode):
    g = load_golden("mixed_2el")
    out = tmp_path / "per_update.csv"
    cmd = [str(CSM), "-q", "query.graph", "-d", "data.graph", "-u", "stream.txt", "-a", algo, "--mode", mode,
           "--batch", "64", "--hash", "1", "--out", str(out)]
    r = subprocess.run(cmd, cwd=g["dir"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    init = json.loads((g["dir"] / "initial.json").read_text())
    k = lines.index("----------- Initial Matching ----------")
    assert lines[k + 2].split()[0] == str(init["graphflow"])
    x = g["exp"]
    assert f"{int(x['symbi_pos'].sum())} positive matches." in lines
    assert f"{int(x['symbi_neg'].sum())} negative matches." in lines
    assert f"{len(g['stream'])} edge updates." in lines
    rows = list(csv.DictReader(open(out)))
    assert np.array_equal(np.array([int(r_["pos"]) for r_ in rows], dtype=np.uint64), x["symbi_pos"])
    assert np.array_equal(np.array([int(r_["neg"]) for r_ in rows], dtype=np.uint64), x["symbi_neg"])
    assert np.array_equal(np.array([int(r_["hash"]) for r_ in rows], dtype=np.uint64), x["symbi_hash"])
    if algo != "parallel_graphflow":
        assert "DAG: " in lines


def test_driver_print_enum_lists_every_embedding():
    g = load_golden("dense_del")
    r = subprocess.run([str(CSM), "-q", "query.graph", "-d", "data.graph", "-u", "stream.txt", "-a", "parallel_symbi",
                        "--print-enum", "1", "--report-initial", "0", "--print-prep", "0"],
                       cwd=g["dir"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    nq = len(g["qv"])
    rows = [ln.split() for ln in r.stdout.splitlines() if ln.strip() and all(t.isdigit() for t in ln.split())]
    rows = [x for x in rows if len(x) == nq]
    x = g["exp"]
    assert len(rows) == int((x["symbi_pos"] + x["symbi_neg"]).sum())


@pytest.mark.parametrize("algo", ["parallel_newsp", "parallel_symbi"])
def test_driver_query_directory_sums_every_query(tmp_path, gen_dir, algo):
    """-q DIR (NewSP's multi-query build): each file is a standing query on the same
    data graph, and each update's counts are the sum over the queries."""
    import shutil

    from oracle import pyoracle
    from paracosm_b200 import workload
    w = workload.generate("c2", gen_dir / f"multiq_{algo}", extra=[
        "--log2-n", "11", "--avg-degree", "6", "--vlabels", "3", "--zipf", "0", "--elabels", "2", "--updates", "300",
        "--insert-frac", "0.8", "--seed", "21", "--query", "5:sparse:1", "--query", "4:dense", "--text"])
    qdir = tmp_path / "queries"
    qdir.mkdir()
    for i in range(2):
        shutil.copy(w.query_path(i), qdir / f"q{i}.graph")
    out = tmp_path / "per_update.csv"
    r = subprocess.run([str(CSM), "-q", str(qdir), "-d", str(w.directory / "data.graph"), "-u",
                        str(w.directory / "stream.txt"), "-a", algo, "--batch", "64", "--out", str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    assert "Load query graph number: 2" in r.stdout
    want_pos = np.zeros(len(w.stream), np.uint64)
    want_neg = np.zeros(len(w.stream), np.uint64)
    for qv, qe in w.queries:
        ref = pyoracle.run(qv, qe, w.vlabels, w.edges, w.stream, want_hash=False)
        want_pos += ref["pos"]
        want_neg += ref["neg"]
    rows = list(csv.DictReader(open(out)))
    assert np.array_equal(np.array([int(x["pos"]) for x in rows], dtype=np.uint64), want_pos)
    assert np.array_equal(np.array([int(x["neg"]) for x in rows], dtype=np.uint64), want_neg)
    assert f"{int(want_pos.sum())} positive matches." in r.stdout.splitlines()
    assert want_pos.sum() > 0
