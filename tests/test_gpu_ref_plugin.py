"""The engine behind the reference's own plugin interface: GpuPlugin
(include/csm_gpu_plugin.h), a subclass of the reference's `matching` class
compiled against its headers, is driven by the reference's sequential update
loop (oracle/_ref/ref_driver_gpu -a gpu_*, the SingleThreadUpdate order of
ParaCOSM/CSM/matching/main.cpp:628-674).  Its per-update counts, and the
match-set hash of the embeddings it prints for --print-enum, must equal the
reference SymBi's recorded in the golden fixtures."""
from __future__ import annotations

import csv
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, golden_cases, load_golden

pytestmark = pytest.mark.gpu

DRIVER = ROOT / "oracle" / "_ref" / "ref_driver_gpu"


def run_driver(d: Path, algo: str, out: Path, cap, homo: bool, want_hash: bool):
    cmd = [str(DRIVER), "-q", str(d / "query.graph"), "-d", str(d / "data.graph"), "-u", str(d / "stream.txt"),
           "-a", algo, "--out", str(out)]
    if cap:
        cmd += ["--max-results", str(cap)]
    if homo:
        cmd += ["--homo", "1"]
    if want_hash:
        cmd += ["--hash"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = list(csv.DictReader(open(out)))
    return (np.array([int(x["pos"]) for x in rows], dtype=np.uint64),
            np.array([int(x["neg"]) for x in rows], dtype=np.uint64),
            np.array([int(x["hash"]) for x in rows], dtype=np.uint64), r.stdout)


@pytest.mark.skipif(not DRIVER.exists(), reason="ref_driver_gpu is built where the reference sources are")
@pytest.mark.parametrize("algo", ["gpu_symbi", "gpu_turboflux", "gpu_graphflow"])
@pytest.mark.parametrize("case", golden_cases())
def test_reference_loop_drives_the_engine_through_class_matching(case, algo, tmp_path):
    g = load_golden(case)
    p = g["params"]
    cap = p["max_results"] or 0
    pos, neg, hsh, stdout = run_driver(g["dir"], algo, tmp_path / "rows.csv", cap, p["homo"], want_hash=True)
    x = g["exp"]
    assert np.array_equal(pos, x["symbi_pos"]), np.nonzero(pos != x["symbi_pos"])[0][:10]
    assert np.array_equal(neg, x["symbi_neg"]), np.nonzero(neg != x["symbi_neg"])[0][:10]
    # hashes of the printed embeddings: every update below the cap (an update that
    # reaches the cap may print more embeddings than it counts)
    ok = (x["symbi_pos"] + x["symbi_neg"] < cap) if cap else np.ones(len(pos), bool)
    assert np.array_equal(hsh[ok], x["symbi_hash"][ok]), np.nonzero(hsh[ok] != x["symbi_hash"][ok])[0][:10]
    assert f"{int(x['symbi_pos'].sum())} positive matches." in stdout
