"""Standing queries sharing one device graph (csm_gpu_attach_query): every
query's per-update results are the same alone (its own engine) and in the
mix (attached to one owner whose submits drive all of them), including
queries attached and detached between submits."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle
from paracosm_b200 import Engine, workload
from paracosm_b200._abi import CSM_EUNSUPPORTED, CsmError

pytestmark = pytest.mark.gpu

QUERIES = ["6:sparse:1", "4:dense", "8:sparse:2", "5:dense"]
PLUGINS = ["parallel_symbi", "parallel_graphflow", "parallel_turboflux", "parallel_symbi"]
CAPS = [0, 0, 5000, 300]


@pytest.fixture(scope="module")
def wl(tmp_path_factory):
    extra = ["--log2-n", "13", "--avg-degree", "10", "--vlabels", "4", "--zipf", "0.8", "--elabels", "2",
             "--updates", "4000", "--insert-frac", "0.75"]
    for q in QUERIES:
        extra += ["--query", q]
    return workload.generate("c2", tmp_path_factory.mktemp("mq") / "w", extra=extra)


def _alone(w, qi, stream, **kw):
    qv, qe = w.queries[qi]
    with Engine(PLUGINS[qi], max_results=CAPS[qi], want_hash=True, **kw) as eng:
        eng.set_query(qv, qe)
        eng.load_graph(w.vlabels, w.edges)
        eng.build_index()
        return eng.run(stream)


def _same(a, b):
    for k in ("pos", "neg", "status", "hash"):
        assert np.array_equal(a[k], b[k]), (k, np.nonzero(a[k] != b[k])[0][:10])


def _owner(w, **kw):
    qv, qe = w.queries[0]
    eng = Engine(PLUGINS[0], max_results=CAPS[0], want_hash=True, **kw)
    eng.set_query(qv, qe)
    eng.reserve_labels(np.unique(w.vlabels), np.unique(w.edges[:, 2]))
    eng.load_graph(w.vlabels, w.edges)
    eng.build_index()
    return eng


@pytest.mark.parametrize("graphs", [False, True])
@pytest.mark.parametrize("max_batch", [65536, 333])
def test_each_query_alone_and_in_the_mix(wl, max_batch, graphs):
    s = wl.stream
    alone = [_alone(wl, i, s, max_batch=max_batch) for i in range(len(QUERIES))]
    with _owner(wl, max_batch=max_batch, graphs=graphs) as own:
        att = [own.attach(*wl.queries[i], PLUGINS[i], max_results=CAPS[i], want_hash=True)
               for i in range(1, len(QUERIES))]
        first = own.submit(s)
        own.wait()
        mixed = [own.results(first, len(s))] + [a.results(first, len(s)) for a in att]
        for i in range(len(QUERIES)):
            _same(mixed[i], alone[i])
        assert sum(int(m["pos"].sum()) for m in mixed) > 0
        for a in att:
            a.close()


def test_attach_and_detach_between_submits(wl):
    s = wl.stream
    cut1, cut2 = 1500, 2800
    alone2 = _alone(wl, 2, s)
    alone3 = _alone(wl, 3, s)
    with _owner(wl) as own:
        own.run(s[:cut1])
        a2 = own.attach(*wl.queries[2], PLUGINS[2], max_results=CAPS[2], want_hash=True)
        first = own.submit(s[cut1:cut2])
        own.wait()
        _same(a2.results(first, cut2 - cut1), alone2[cut1:cut2])
        a3 = own.attach(*wl.queries[3], PLUGINS[3], max_results=CAPS[3], want_hash=True)
        a2.close()
        first = own.submit(s[cut2:])
        own.wait()
        _same(a3.results(first, len(s) - cut2), alone3[cut2:])
        # an attached query's index follows the shared graph
        ix = a3.index(len(wl.vlabels))
        want = pyoracle.index(*wl.queries[3], wl.vlabels, wl.edges, s, algo="symbi")
        assert np.array_equal(ix["d1"][:, :len(wl.vlabels)], want["d1"])
        assert np.array_equal(ix["d2"][:, :len(wl.vlabels)], want["d2"])
        assert a3.initial_match() == pyoracle.initial_count(*wl.queries[3], wl.vlabels, wl.edges, s)
        a3.close()


def test_attaching_a_query_with_labels_the_owner_folded_away(wl):
    qv, qe = wl.queries[0]
    with Engine(PLUGINS[0]) as own:
        own.set_query(qv, qe)
        own.load_graph(wl.vlabels, wl.edges)
        own.build_index()
        other = np.full(3, 1000, dtype=np.uint32)
        with pytest.raises(CsmError) as e:
            own.attach(other, np.array([(0, 1, 0), (1, 2, 0)], dtype=np.uint32))
        assert e.value.code == CSM_EUNSUPPORTED
