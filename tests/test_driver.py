"""The csm driver (paracosm_b200/_bin/csm): the reference's command line and
output lines over the engine.  CPU checks here; the GPU run is in
test_gpu_driver.py."""
from __future__ import annotations

import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
CSM = ROOT / "paracosm_b200" / "_bin" / "csm"
GOLD = Path(__file__).resolve().parent / "golden" / "c1_small"


def test_help_lists_the_reference_options():
    r = subprocess.run([str(CSM), "-h"], capture_output=True, text=True)
    assert r.returncode == 0
    for opt in ("-q", "-d", "-u", "-a", "--max-results", "--time-limit", "--print-prep", "--print-enum", "--homo",
                "--report-initial", "--initial-time-limit", "--orders", "--auto-tuning"):
        assert opt in r.stderr


def test_missing_required_options_fail_without_touching_the_gpu():
    r = subprocess.run([str(CSM), "-q", "x"], capture_output=True, text=True)
    assert r.returncode == 2 and "required" in r.stderr


def test_unknown_algorithm_is_reported_like_the_reference():
    r = subprocess.run([str(CSM), "-q", "query.graph", "-d", "data.graph", "-u", "stream.txt", "-a", "nope"],
                       cwd=GOLD, capture_output=True, text=True)
    assert r.returncode == 1
    assert "----------- Loading graphs ------------" in r.stdout and "Unknown algorithm" in r.stdout
    assert "# vertices = 2048" in r.stdout


def test_serve_tool_usage():
    serve = ROOT / "paracosm_b200" / "_bin" / "csm_serve"
    r = subprocess.run([str(serve), "-h"], capture_output=True, text=True)
    assert r.returncode == 0
    for opt in ("-w", "--rate", "--max-batch", "--budget-gb", "--arrive-every", "--out"):
        assert opt in r.stderr
    r = subprocess.run([str(serve)], capture_output=True, text=True)
    assert r.returncode == 2


def test_loaders_drop_self_loops_and_duplicate_edges(tmp_path):
    """Edges are kept once, the first occurrence winning (Graph::AddEdge is a no-op on an
    existing edge, ParaCOSM/CSM/graph/graph.cpp:63-64); self loops are dropped.  The csm
    driver prints the loaded sizes before it needs a GPU."""
    (tmp_path / "q").write_text("v 0 0\nv 1 0\ne 0 1 0\n")
    (tmp_path / "d").write_text("v 0 0\nv 1 0\nv 2 0\ne 0 1 5\ne 1 0 6\ne 1 2 0\ne 2 2 0\ne 0 1 7\ne 2 0 1\n")
    (tmp_path / "s").write_text("e 0 2 0\n")
    r = subprocess.run([str(CSM), "-q", str(tmp_path / "q"), "-d", str(tmp_path / "d"), "-u", str(tmp_path / "s"),
                        "-a", "parallel_symbi"], capture_output=True, text=True, timeout=120)
    sizes = [ln for ln in r.stdout.splitlines() if ln.startswith("# edges = ")]
    assert sizes[:2] == ["# edges = 1", "# edges = 3"], r.stdout


def test_malformed_option_values_print_usage():
    for tool, args in ((CSM, ["-q", "a", "-d", "b", "-u", "c", "--max-results", "many"]),
                       (CSM.parent / "calig", ["-d", "a", "-q", "b", "-s", "c", "-c", "x"])):
        r = subprocess.run([str(tool)] + args, capture_output=True, text=True, timeout=60)
        assert r.returncode == 2
        assert "bad option value" in r.stderr
