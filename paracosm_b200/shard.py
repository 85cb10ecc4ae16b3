"""Seed sharding across GPUs: one process per GPU, each holding a replica of
the data graph and applying every batch, each searching only its share of the
root tasks (csm_cfg.shard_rank / shard_count).  The per-update results of all
shards combine into the unsharded results: counts, match-set hashes and
algorithmic bytes add up, the cap applies to the sum, an update is INVALID
everywhere or nowhere, TIMED_OUT if any shard ran out of time, and its
latency is the slowest shard's.

`combine` does this on host arrays; `allreduce_results` does it across the
ranks of a torch.distributed process group (gloo on CPU tensors, NCCL on
device tensors), with the results viewed as an [n, 6] int64 tensor (the
48-byte csm_result records).
"""
from __future__ import annotations

import numpy as np

from ._abi import RESULT_DTYPE, ST_CAPPED, ST_INVALID, ST_OK, ST_TIMED_OUT


def combine(parts: list[np.ndarray], cap: int = 0) -> np.ndarray:
    """Per-update results of every shard (same updates, same order) -> unsharded results."""
    out = parts[0].copy()
    with np.errstate(over="ignore"):
        for k in ("pos", "neg", "hash", "work_bytes"):
            out[k] = np.sum([p[k] for p in parts], axis=0, dtype=np.uint64)
    out["latency_ns"] = np.max([p["latency_ns"] for p in parts], axis=0)
    invalid = np.any([p["status"] == ST_INVALID for p in parts], axis=0)
    timed = np.any([p["status"] == ST_TIMED_OUT for p in parts], axis=0)
    total = out["pos"] + out["neg"]
    capped = (total >= cap) if cap else np.zeros(len(out), dtype=bool)
    if cap:
        out["pos"] = np.minimum(out["pos"], np.uint64(cap))
        out["neg"] = np.minimum(out["neg"], np.uint64(cap))
    status = np.full(len(out), ST_OK, dtype=np.uint32)
    status[timed & ~capped] = ST_TIMED_OUT
    status[capped] = ST_CAPPED
    status[invalid] = ST_INVALID
    out["status"] = status
    out["hash"][status != ST_OK] = 0
    return out


def allreduce_results(t, cap: int = 0, group=None):
    """In place on every rank: t is the int64 [n, 6] view of this rank's csm_result records
    (pos, neg, hash, work_bytes, latency_ns, status | safe << 32); afterwards it holds the
    combined results.  Three collectives: a sum, a sum of status indicators, a max."""
    import torch
    import torch.distributed as dist

    status = t[:, 5] & 0xFFFFFFFF
    safe = t[:, 5] >> 32
    sums = t[:, 0:4].clone()
    flags = torch.stack([(status == ST_INVALID).to(torch.int64), (status == ST_TIMED_OUT).to(torch.int64)], dim=1)
    lat = t[:, 4].clone()
    dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(flags, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(lat, op=dist.ReduceOp.MAX, group=group)
    pos, neg, hsh, work = sums[:, 0], sums[:, 1], sums[:, 2], sums[:, 3]
    capped = (pos + neg >= cap) if cap else torch.zeros_like(pos, dtype=torch.bool)
    if cap:
        pos = torch.clamp(pos, max=cap)
        neg = torch.clamp(neg, max=cap)
    st = torch.full_like(pos, ST_OK)
    st = torch.where((flags[:, 1] > 0) & ~capped, torch.full_like(st, ST_TIMED_OUT), st)
    st = torch.where(capped, torch.full_like(st, ST_CAPPED), st)
    st = torch.where(flags[:, 0] > 0, torch.full_like(st, ST_INVALID), st)
    hsh = torch.where(st == ST_OK, hsh, torch.zeros_like(hsh))
    t[:, 0] = pos
    t[:, 1] = neg
    t[:, 2] = hsh
    t[:, 3] = work
    t[:, 4] = lat
    t[:, 5] = st | (safe << 32)
    return t


def as_int64_rows(res: np.ndarray) -> np.ndarray:
    """Host results (RESULT_DTYPE) as the [n, 6] int64 rows allreduce_results works on."""
    assert res.dtype == RESULT_DTYPE
    return np.ascontiguousarray(res).view(np.int64).reshape(-1, 6)
