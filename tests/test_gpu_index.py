"""GPU candidate index (TurboFlux DCG / SymBi DCS as device bitsets) against the
reference plugins' own index state (golden fixtures read out of the plugin
objects) and against the oracle's restatement, after whole batches."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases, load_golden, load_golden_index
from oracle import pyoracle
from paracosm_b200 import UPDATE_DTYPE, Engine, workload

pytestmark = pytest.mark.gpu


def _engine(algo, g, **kw):
    eng = Engine(algo, **kw)
    eng.set_query(g["qv"], g["qe"])
    eng.load_graph(g["vl"], g["e"])
    eng.build_index()
    return eng


def _same_index(got, want, n):
    assert got["root"] == want["root"]
    assert got["order"] == want["order"]
    assert got["parents"] == want["parents"]
    assert np.array_equal(got["d1"][:, :n], want["d1"][:, :n]), np.argwhere(got["d1"][:, :n] != want["d1"][:, :n])[:8]
    assert np.array_equal(got["d2"][:, :n], want["d2"][:, :n]), np.argwhere(got["d2"][:, :n] != want["d2"][:, :n])[:8]
    assert not got["d1"][:, n:].any() and not got["d2"][:, n:].any()


@pytest.mark.parametrize("max_batch", [65536, 7])
@pytest.mark.parametrize("algo", ["symbi", "turboflux"])
@pytest.mark.parametrize("case", golden_cases())
def test_index_equals_the_reference_plugins_index(case, algo, max_batch):
    g = load_golden(case)
    ref = load_golden_index(case, algo)
    n = len(g["vl"])
    ats = sorted(ref)
    with _engine("parallel_" + algo, g, max_batch=max_batch) as eng:
        _same_index(eng.index(), ref[ats[0]], n)
        for a, b in zip(ats, ats[1:]):
            eng.run(g["stream"][a:b])
            _same_index(eng.index(), ref[b], n)


@pytest.mark.parametrize("algo", ["symbi", "turboflux"])
def test_index_after_every_plain_update_matches_the_oracle(algo):
    g = load_golden("dense_del")
    n = len(g["vl"])
    s = g["stream"]
    with _engine("parallel_" + algo, g, mode="plain") as eng:
        for k in range(0, 60, 3):
            eng.run(s[k:k + 3])
            want = pyoracle.index(g["qv"], g["qe"], g["vl"], g["e"], s[:k + 3], algo=algo)
            _same_index(eng.index(), want, n)


@pytest.mark.parametrize("algo", ["symbi", "turboflux"])
def test_index_with_deletions_across_many_batches(gen_dir, algo):
    w = workload.generate("c2", gen_dir / f"ixdel_{algo}", extra=["--log2-n", "13", "--updates", "3000",
                                                                   "--insert-frac", "0.6"])
    qv, qe = w.queries[0]
    n = len(w.vlabels)
    cuts = [0, 1, 700, 701, 1900, 3000]
    with Engine("parallel_" + algo, max_batch=256) as eng:
        eng.set_query(qv, qe)
        eng.load_graph(w.vlabels, w.edges)
        eng.build_index()
        for a, b in zip(cuts, cuts[1:]):
            eng.run(w.stream[a:b])
            want = pyoracle.index(qv, qe, w.vlabels, w.edges, w.stream[:b], algo=algo)
            _same_index(eng.index(), want, n)


def test_index_after_vertex_insertion():
    vl = np.array([0, 1, 0, 1], dtype=np.uint32)
    edges = np.array([(0, 1, 0), (1, 2, 0), (2, 3, 0)], dtype=np.uint32)
    qv = np.array([0, 1, 0], dtype=np.uint32)
    qe = np.array([(0, 1, 0), (1, 2, 0)], dtype=np.uint32)
    ups = np.array([(ord("v"), 1, 0, 4, 0, 0), (ord("e"), 1, 0, 4, 1, 0), (ord("e"), 1, 0, 4, 3, 0),
                    (ord("v"), 1, 0, 5, 1, 0)], dtype=UPDATE_DTYPE)
    for algo in ("symbi", "turboflux"):
        with Engine("parallel_" + algo, vertex_headroom=16) as eng:
            eng.set_query(qv, qe)
            eng.load_graph(vl, edges)
            eng.build_index()
            for k in range(len(ups)):
                eng.run(ups[k:k + 1])
                want = pyoracle.index(qv, qe, vl, edges, ups[:k + 1], algo=algo)
                _same_index(eng.index(), want, len(want["d1"][0]))


def test_index_counts_in_stats():
    g = load_golden("zipf_8q")
    with _engine("parallel_symbi", g) as eng:
        ix = eng.index()
        st = eng.stats()
        assert st["index_entries"] == ix["d1"].sum() == ix["d1_count"]
        assert st["index_vertices"] == ix["d2"].sum() == ix["d2_count"]
