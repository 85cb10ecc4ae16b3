"""Shared test setup: the `gpu` marker and the golden-fixture loader."""
from __future__ import annotations

import csv
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


def golden_cases() -> list[str]:
    return sorted(d.name for d in GOLDEN.iterdir() if d.is_dir() and (d / "expected.csv").exists())


def load_golden(name: str) -> dict:
    from paracosm_b200 import workload
    d = GOLDEN / name
    params = json.loads((d / "params.json").read_text())
    qv, qe = workload.read_graph(d / "query.graph")
    vl, e = workload.read_graph(d / "data.graph")
    s = workload.read_stream(d / "stream.txt")
    rows = list(csv.DictReader(open(d / "expected.csv")))
    exp = {}
    for col in rows[0].keys():
        if col == "idx":
            continue
        exp[col] = np.array([int(r[col]) if r[col] != "" else 0 for r in rows], dtype=np.uint64)
    return {"dir": d, "params": params, "qv": qv, "qe": qe, "vl": vl, "e": e, "stream": s, "exp": exp}


@pytest.fixture(scope="session")
def gen_dir(tmp_path_factory):
    return tmp_path_factory.mktemp("workloads")
