"""csm_gpu_probe_noalloc, the entry point for callers that cannot allocate
device memory where they need counts (a locked or stream-ordered memory pool,
a latency-critical loop in which an allocation would synchronise the device).

It reads the graph an existing context holds and keeps its working memory in
a static device array.  Its counts must equal what the ordinary entry point
reports for the same edges: an insertion of an edge that is already in the
graph counts the embeddings containing it and leaves the graph unchanged.
The counts are also checked against the oracle's count for an insertion of
each edge.  For the CaLiG-style plugin such an insertion counts 0 (its rule for
a present edge), which the probe must report as well.  Two calls in a row check
that the shared array is cleared between calls, and several contexts with
different queries check that one array serves them all.
This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from paracosm_b200 import UPDATE_DTYPE, Engine

pytestmark = pytest.mark.gpu


def _edges_present_after(g) -> dict:
    cur = {(min(int(a), int(b)), max(int(a), int(b))): int(l) for a, b, l in g["e"]}
    for u in g["stream"]:
        k = (min(int(u["id1"]), int(u["id2"])), max(int(u["id1"]), int(u["id2"])))
        if u["is_add"]:
            cur.setdefault(k, int(u["label"]))
        else:
            cur.pop(k, None)
    return cur


@pytest.mark.parametrize("case,algo", [("c1_small", "parallel_graphflow"), ("mixed_2el", "parallel_symbi"),
                                       ("zipf_8q", "parallel_turboflux"), ("dense_del", "parallel_calig")])
def test_probe_noalloc_matches_the_submit_path_on_two_calls(case, algo):
    import torch

    from oracle import pyoracle

    g = load_golden(case)
    with Engine(algo) as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        eng.run(g["stream"])
        cur = _edges_present_after(g)
        keys = sorted(cur)[:: max(1, len(cur) // 700)][:1000]
        ups = np.zeros(len(keys), dtype=UPDATE_DTYPE)
        for i, (a, b) in enumerate(keys):
            ups[i] = (ord("e"), 1, 0, a, b, cur[(a, b)])
        d_edges = torch.from_numpy(ups.view(np.uint8).copy()).cuda()
        # the oracle's count for an insertion of each present edge (the graph does not change)
        orc = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], np.concatenate([g["stream"], ups]),
                           want_hash=False)["pos"][len(g["stream"]):]
        if algo == "parallel_calig":
            orc = np.zeros_like(orc)  # CaLiG: an insertion of a present edge counts 0
        for call in range(2):
            d_counts = torch.full((len(ups),), -1, dtype=torch.int64, device="cuda")
            rc = eng.lib.csm_gpu_probe_noalloc(eng.h, len(ups), d_edges.data_ptr(), d_counts.data_ptr())
            assert rc == 0, eng.lib.csm_gpu_last_error()
            probe = d_counts.cpu().numpy().astype(np.uint64)
            ref = eng.run(ups)  # insertions of present edges: counted, graph unchanged
            assert np.array_equal(probe, ref["pos"]), (call, np.nonzero(probe != ref["pos"])[0][:10])
            assert np.array_equal(probe, orc), (call, np.nonzero(probe != orc)[0][:10])
            if algo != "parallel_calig":
                assert probe.sum() > 0


def test_probe_noalloc_rejects_more_than_its_maximum():
    import torch

    g = load_golden("c1_small")
    with Engine("parallel_graphflow") as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        d_edges = torch.zeros(1025 * UPDATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        d_counts = torch.zeros(1025, dtype=torch.int64, device="cuda")
        rc = eng.lib.csm_gpu_probe_noalloc(eng.h, 1025, d_edges.data_ptr(), d_counts.data_ptr())
        assert rc == -1
        assert b"at most 1024" in eng.lib.csm_gpu_last_error()


def test_probe_noalloc_on_an_attached_query_reads_the_graph_after_the_owners_submit():
    """An attached query's graph belongs to its owner, whose submits mutate it on the owner's
    stream: a probe right after an owner submit (without waiting) must see that submit's edges."""
    import torch

    from oracle import pyoracle

    g = load_golden("mixed_2el")
    with Engine("parallel_graphflow") as own:
        own.set_query(g["qv"], g["qe"])
        own.reserve_labels(np.unique(g["qv"]), np.unique(g["qe"][:, 2]))
        own.load_graph(g["vl"], g["e"])
        own.build_index()
        att = own.attach(g["qv"], g["qe"], "parallel_graphflow")
        own.submit(g["stream"])  # no wait: the probe is ordered after it on the device
        cur = _edges_present_after(g)
        ins = [k for k, u in zip(range(len(g["stream"])), g["stream"]) if u["is_add"]]
        keys = []
        for i in ins:
            u = g["stream"][i]
            k = (min(int(u["id1"]), int(u["id2"])), max(int(u["id1"]), int(u["id2"])))
            if k in cur and k not in keys:
                keys.append(k)
        keys = keys[:500]
        ups = np.zeros(len(keys), dtype=UPDATE_DTYPE)
        for i, (a, b) in enumerate(keys):
            ups[i] = (ord("e"), 1, 0, a, b, cur[(a, b)])
        d_edges = torch.from_numpy(ups.view(np.uint8).copy()).cuda()
        d_counts = torch.full((len(ups),), -1, dtype=torch.int64, device="cuda")
        rc = att.lib.csm_gpu_probe_noalloc(att.h, len(ups), d_edges.data_ptr(), d_counts.data_ptr())
        assert rc == 0, att.lib.csm_gpu_last_error()
        probe = d_counts.cpu().numpy().astype(np.uint64)
        orc = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], np.concatenate([g["stream"], ups]),
                           want_hash=False)["pos"][len(g["stream"]):]
        assert np.array_equal(probe, orc), np.nonzero(probe != orc)[0][:10]
        assert probe.sum() > 0
        own.wait()
