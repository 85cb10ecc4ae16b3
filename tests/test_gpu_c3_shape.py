"""GPU parity on the shape of the 2^22-vertex SymBi benchmark, at 2^16 vertices: a
16-vertex dense query, 16 vertex labels Zipf(1.2), 4 edge labels, an 80/20 stream
of 70,000 updates in batches of up to 65,536.  Every per-update count, status and
match-set hash is compared, through the C ABI, with the reference's sequential
SymBi (tests/golden/c3_shape, recorded with max_results 1e6 and 20,000), with the
independent tail counted and enumerated, and one update per launch on a prefix."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_c3_shape
from paracosm_b200 import ST_CAPPED, ST_OK, Engine

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c3s(tmp_path_factory):
    return load_c3_shape(tmp_path_factory.mktemp("c3_shape"))


def run(c, n=None, **kw):
    w = c["w"]
    qv, qe = w.queries[0]
    s = w.stream if n is None else w.stream[:n]
    with Engine(kw.pop("algo", "parallel_symbi"), **kw) as eng:
        eng.set_query(qv, qe)
        eng.load_graph(w.vlabels, w.edges)
        eng.build_index()
        return eng.run(s)


def check(res, pos, neg, cap):
    n = len(res)
    bad = np.nonzero((res["pos"] != pos[:n]) | (res["neg"] != neg[:n]))[0]
    assert len(bad) == 0, [(int(i), int(res["pos"][i]), int(res["neg"][i]), int(pos[i]), int(neg[i]))
                           for i in bad[:5]]
    assert np.array_equal(res["status"] == ST_CAPPED, (pos[:n] + neg[:n]) >= cap)
    assert not np.any((res["status"] != ST_OK) & (res["status"] != ST_CAPPED))


@pytest.mark.parametrize("algo", ["parallel_symbi", "parallel_turboflux", "parallel_graphflow"])
@pytest.mark.parametrize("tail_enumerate", [False, True])
def test_c3_shape_batched_counts(c3s, tail_enumerate, algo):
    x = c3s["exp"]
    cap = c3s["params"]["max_results"]
    res = run(c3s, algo=algo, max_results=cap, max_batch=65536, tail_enumerate=tail_enumerate)
    check(res, x["pos"], x["neg"], cap)
    assert int(((res["pos"] + res["neg"]) > 0).sum()) == 56


def test_c3_shape_batched_hashes(c3s):
    x = c3s["exp"]
    cap = c3s["params"]["max_results"]
    res = run(c3s, max_results=cap, max_batch=65536, want_hash=True)
    check(res, x["pos"], x["neg"], cap)
    assert np.array_equal(res["hash"], x["hash"])


@pytest.mark.parametrize("tail_enumerate", [False, True])
def test_c3_shape_capped(c3s, tail_enumerate):
    x = c3s["exp"]
    cap = c3s["params"]["max_results_capped"]
    res = run(c3s, max_results=cap, max_batch=65536, tail_enumerate=tail_enumerate)
    check(res, x["cap_pos"], x["cap_neg"], cap)
    assert int((res["status"] == ST_CAPPED).sum()) > 0


def test_c3_shape_one_update_per_launch(c3s):
    x = c3s["exp"]
    cap = c3s["params"]["max_results"]
    res = run(c3s, n=5000, max_results=cap, mode="plain")
    check(res, x["pos"], x["neg"], cap)
    assert int(((res["pos"] + res["neg"]) > 0).sum()) == 3
