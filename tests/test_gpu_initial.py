"""GPU InitialMatching (csm_gpu_initial_match) against the counts the reference's
own csm driver prints (golden initial.json) and against the oracle after updates."""
from __future__ import annotations

import json

import pytest

from conftest import golden_cases, load_golden
from oracle import pyoracle
from paracosm_b200 import Engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algo", ["parallel_graphflow", "parallel_turboflux", "parallel_symbi"])
@pytest.mark.parametrize("case", golden_cases())
def test_initial_match_equals_the_reference(case, algo):
    g = load_golden(case)
    want = json.loads((g["dir"] / "initial.json").read_text())
    # a 1000-seed batch forces several search launches on the larger cases
    with Engine(algo, homo=g["params"]["homo"], max_batch=1000,
                max_results=g["params"]["max_results"] or 0) as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        assert eng.initial_match() == want[algo.split("_")[1]]


def test_initial_match_after_updates():
    g = load_golden("dense_del")
    s = g["stream"]
    with Engine("parallel_symbi") as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        for a, b in ((0, 100), (100, 300)):
            eng.run(s[a:b])
            assert eng.initial_match() == pyoracle.initial_count(g["qv"], g["qe"], g["vl"], g["e"], s[:b])
