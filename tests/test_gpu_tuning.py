"""Autotuner (csm_gpu_autotune): picks an admissible launch shape from timings
on sample edges, leaves the graph untouched, and the counts afterwards are
unchanged."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from paracosm_b200 import Engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algo", ["parallel_graphflow", "parallel_symbi"])
def test_autotune_keeps_results_and_graph(algo):
    g = load_golden("zipf_8q")
    with Engine(algo, want_hash=True) as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        before = eng.initial_match()
        shape = eng.autotune(g["stream"][:200])
        assert shape["warps_per_block"] in (4, 8, 16)
        assert 1 <= shape["blocks_per_sm"] and shape["warps_per_block"] * shape["blocks_per_sm"] <= 32
        assert shape["sample_search_ms"] > 0
        assert shape["donate_every"] in (0, 1, 2, 4) and shape["split_deep"] in (0, 16, 64, 256)
        assert eng.initial_match() == before  # the sample did not touch the graph
        res = eng.run(g["stream"])
        x = g["exp"]
        assert np.array_equal(res["pos"], x["symbi_pos"]) and np.array_equal(res["neg"], x["symbi_neg"])
        assert np.array_equal(res["hash"], x["symbi_hash"])
