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
