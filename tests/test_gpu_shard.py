"""Seed sharding on the device: the shards of a stream, run one after another
on one GPU (each a full replica that searches only its root tasks), combine
into exactly the unsharded per-update results.  No shard waits on another."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from oracle import pyoracle
from paracosm_b200 import Engine
from paracosm_b200.shard import combine

pytestmark = pytest.mark.gpu


def _run(g, algo, shards, rank, cap, **kw):
    with Engine(algo, max_results=cap, want_hash=True, shard_rank=rank, shard_count=shards, **kw) as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        res = eng.run(g["stream"])
        init = eng.initial_match()
    return res, init


@pytest.mark.parametrize("shards", [2, 3])
@pytest.mark.parametrize("case,algo", [("mixed_2el", "parallel_symbi"), ("capped", "parallel_turboflux"),
                                       ("zipf_8q", "parallel_graphflow")])
def test_shards_combine_to_the_unsharded_results(case, algo, shards):
    g = load_golden(case)
    cap = g["params"]["max_results"] or 0
    full, full_init = _run(g, algo, 1, 0, cap)
    parts = [_run(g, algo, shards, r, cap) for r in range(shards)]
    out = combine([p[0] for p in parts], cap)
    for k in ("pos", "neg", "status", "hash"):
        assert np.array_equal(out[k], full[k]), (k, np.nonzero(out[k] != full[k])[0][:10])
    if not cap:
        assert np.array_equal(out["work_bytes"], full["work_bytes"])
    assert sum(p[1] for p in parts) == full_init
    x = g["exp"]
    assert np.array_equal(out["pos"], x["symbi_pos"]) and np.array_equal(out["neg"], x["symbi_neg"])


def test_shard_rank_outside_the_count_is_refused():
    from paracosm_b200._abi import CSM_EINVAL, CsmError
    with pytest.raises(CsmError) as e:
        Engine("parallel_symbi", shard_rank=2, shard_count=2)
    assert e.value.code == CSM_EINVAL
