"""Seed sharding across GPUs, host side: combining per-shard results, on host
arrays and across a world-size-2 gloo process group on CPU."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from paracosm_b200 import RESULT_DTYPE, ST_CAPPED, ST_INVALID, ST_OK, ST_TIMED_OUT
from paracosm_b200.shard import allreduce_results, as_int64_rows, combine


def _parts(n=500, shards=2, cap=1000, seed=3):
    """Exact per-update results split across shards the way the engine splits seeds."""
    rng = np.random.default_rng(seed)
    full = rng.integers(0, 1500, n).astype(np.uint64)
    full[rng.random(n) < 0.3] = 0
    is_add = rng.random(n) < 0.8
    invalid = rng.random(n) < 0.05
    timed = rng.random(n) < 0.05
    hashes = rng.integers(0, 2**63, (shards, n), dtype=np.int64).astype(np.uint64)
    split = np.zeros((shards, n), dtype=np.uint64)
    for i in range(n):
        cuts = np.sort(rng.integers(0, int(full[i]) + 1, shards - 1))
        split[:, i] = np.diff(np.concatenate([[0], cuts, [full[i]]]))
    parts = []
    for r in range(shards):
        p = np.zeros(n, dtype=RESULT_DTYPE)
        c = np.minimum(split[r], cap) if cap else split[r]
        p["pos"] = np.where(is_add & ~invalid, c, 0)
        p["neg"] = np.where(~is_add & ~invalid, c, 0)
        p["status"] = np.where(invalid, ST_INVALID, np.where(cap and (split[r] >= cap), ST_CAPPED, ST_OK))
        p["status"][(r == 0) & timed & (p["status"] == ST_OK)] = ST_TIMED_OUT
        p["hash"] = np.where(p["status"] == ST_OK, hashes[r], 0)
        p["work_bytes"] = split[r] * 4
        p["latency_ns"] = rng.integers(1, 10**6, n)
        p["safe"] = (full == 0).astype(np.uint32)
        parts.append(p)
    return parts, full, is_add, invalid, timed, hashes


def test_combine_follows_the_unsharded_semantics():
    cap = 1000
    parts, full, is_add, invalid, timed, hashes = _parts(cap=cap)
    out = combine(parts, cap)
    total = np.where(invalid, 0, np.minimum(full, cap))
    assert np.array_equal(out["pos"] + out["neg"], total)
    assert np.all(out["status"][invalid] == ST_INVALID)
    capped = ~invalid & (full >= cap)
    assert np.all(out["status"][capped] == ST_CAPPED)
    assert np.all(out["status"][~invalid & ~capped & timed] == ST_TIMED_OUT)
    ok = out["status"] == ST_OK
    with np.errstate(over="ignore"):
        assert np.array_equal(out["hash"][ok], (hashes[0] + hashes[1])[ok])
    assert np.all(out["hash"][~ok] == 0)
    assert np.array_equal(out["latency_ns"], np.maximum(parts[0]["latency_ns"], parts[1]["latency_ns"]))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts, *_ = _parts(shards=world, cap=1000)
        t = torch.from_numpy(as_int64_rows(parts[rank]).copy())
        allreduce_results(t, cap=1000)
        got = t.numpy().copy().view(RESULT_DTYPE).reshape(-1)
        want = combine(parts, 1000)
        ok = all(np.array_equal(got[k], want[k]) for k in ("pos", "neg", "hash", "work_bytes", "latency_ns",
                                                            "status", "safe"))
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


def test_allreduce_results_on_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got == {0: True, 1: True}
    assert all(p.exitcode == 0 for p in procs)
