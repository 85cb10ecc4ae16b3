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
    """Fixtures that store their inputs in the reference's text formats."""
    return sorted(d.name for d in GOLDEN.iterdir()
                  if d.is_dir() and (d / "expected.csv").exists() and (d / "data.graph").exists())


def load_c3_shape(out_dir: Path) -> dict:
    """The c3_shape case: its inputs rebuilt by the seeded generator (checked against the
    SHA-256 recorded with the fixture) and the reference SymBi's per-update counts, as full
    arrays over the stream (updates not listed in expected.csv count 0)."""
    import hashlib
    import subprocess

    from paracosm_b200 import workload
    d = GOLDEN / "c3_shape"
    params = json.loads((d / "params.json").read_text())
    if not (out_dir / "stream.bin").exists():
        subprocess.run([str(ROOT / "paracosm_b200" / "_bin" / "csm_gen")] + params["generator"] +
                       ["--out", str(out_dir)], check=True, capture_output=True)
    for f, h in params["sha256"].items():
        got = hashlib.sha256((out_dir / f).read_bytes()).hexdigest()
        assert got == h, f"the generator no longer writes the c3_shape inputs: {f} differs"
    w = workload.load(out_dir)
    n = params["updates"]
    assert len(w.stream) == n
    exp = {k: np.zeros(n, dtype=np.uint64) for k in ("pos", "neg", "hash", "cap_pos", "cap_neg")}
    for r in csv.DictReader(open(d / "expected.csv")):
        i = int(r["idx"])
        exp["pos"][i], exp["neg"][i], exp["hash"][i] = int(r["symbi_pos"]), int(r["symbi_neg"]), int(r["symbi_hash"])
        exp["cap_pos"][i], exp["cap_neg"][i] = int(r["symbi_cap_pos"]), int(r["symbi_cap_neg"])
    return {"w": w, "params": params, "exp": exp}


def calig_cases() -> list[str]:
    """Fixtures in the reference CaLiG program's formats, with its per-update counts."""
    return sorted(d.name for d in GOLDEN.iterdir() if d.is_dir() and (d / "expected.txt").exists())


def load_calig(name: str) -> dict:
    from paracosm_b200 import workload
    d = GOLDEN / name
    qv, qe = workload.read_calig_graph(d / "query")
    vl, e = workload.read_calig_graph(d / "data")
    s = workload.read_calig_stream(d / "stream")
    exp = np.loadtxt(d / "expected.txt", dtype=np.uint64).reshape(-1)
    lit_pairs = np.loadtxt(d / "lit.txt", dtype=np.int64).reshape(-1, 2)
    lit = np.zeros((len(qv), len(vl)), dtype=bool)
    lit[lit_pairs[:, 0], lit_pairs[:, 1]] = True
    return {"dir": d, "qv": qv, "qe": qe, "vl": vl, "e": e, "stream": s, "exp": exp, "lit": lit}


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


def load_golden_index(name: str, algo: str) -> dict:
    """The reference plugin's own index state ({update count: {root, order, parents, d1, d2}}),
    with d1 / d2 as bool arrays [n_qv, n_vertices]."""
    d = GOLDEN / name
    n = len(load_golden(name)["vl"])
    out: dict = {}
    cur = None
    for line in (d / f"index_{algo}.txt").read_text().splitlines():
        t = line.split()
        if t[0] == "at":
            cur = {"parents": [], "d1": [], "d2": []}
            out[int(t[1])] = cur
        elif t[0] == "root":
            cur["root"] = int(t[1])
        elif t[0] == "order":
            cur["order"] = [int(x) for x in t[1:]]
        elif t[0] == "parents":
            cur["parents"].append([int(x) for x in t[2:]])
        else:
            bits = np.unpackbits(np.frombuffer(bytes.fromhex(t[2]), dtype=np.uint8), bitorder="little")
            cur[t[0]].append(bits[:n].astype(bool))
    for cur in out.values():
        cur["d1"] = np.array(cur["d1"])
        cur["d2"] = np.array(cur["d2"])
    return out


@pytest.fixture(scope="session")
def gen_dir(tmp_path_factory):
    return tmp_path_factory.mktemp("workloads")
