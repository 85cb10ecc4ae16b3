"""ctypes front end of the CPU restatement (oracle/csm_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker and the CPU baseline, never the product.
"""
from __future__ import annotations

import csv
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
LIB = ROOT / "_build" / "libcsm_oracle.so"
REF_DRIVER = ROOT / "_ref" / "ref_driver"

UPDATE_DTYPE = np.dtype(
    [("type", "u1"), ("is_add", "u1"), ("pad", "<u2"), ("id1", "<u4"), ("id2", "<u4"), ("label", "<u4")]
)
ORACLE_RESULT = np.dtype(
    [("pos", "<u8"), ("neg", "<u8"), ("hash", "<u8"), ("bytes", "<u8"), ("status", "<u4"), ("safe", "<u4")]
)
ST_OK, ST_CAPPED, ST_INVALID = 0, 1, 3

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            subprocess.run(["make", "-C", str(ROOT)], check=True, capture_output=True)
        _lib = C.CDLL(str(LIB))
        _lib.oracle_run.restype = C.c_int
        _lib.oracle_run.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                    C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_int, C.c_int,
                                    C.c_void_p]
        _lib.oracle_brute_count.restype = C.c_int
        _lib.oracle_brute_count.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                            C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32, C.c_int,
                                            C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        _lib.oracle_graphflow_orders.restype = C.c_int
        _lib.oracle_graphflow_orders.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


def run(q_vlabels, q_edges, vlabels, edges, updates, *, max_results: int = 0, homo: bool = False,
        want_hash: bool = True) -> np.ndarray:
    """Per-update (pos, neg, hash, bytes, status, safe) in stream order."""
    qv = np.ascontiguousarray(q_vlabels, dtype=np.uint32)
    qe = np.ascontiguousarray(q_edges, dtype=np.uint32).reshape(-1, 3)
    vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
    e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 3)
    u = np.ascontiguousarray(updates, dtype=UPDATE_DTYPE)
    out = np.zeros(len(u), dtype=ORACLE_RESULT)
    rc = lib().oracle_run(len(qv), _p(qv), len(qe), _p(qe), len(vl), _p(vl), len(e), _p(e), len(u), _p(u),
                          int(max_results), int(homo), int(want_hash), _p(out))
    if rc != 0:
        raise RuntimeError(f"oracle_run failed: {rc}")
    return out


def brute_count(q_vlabels, q_edges, vlabels, edges, v1: int, v2: int, homo: bool = False) -> tuple[int, int]:
    qv = np.ascontiguousarray(q_vlabels, dtype=np.uint32)
    qe = np.ascontiguousarray(q_edges, dtype=np.uint32).reshape(-1, 3)
    vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
    e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 3)
    c, h = C.c_uint64(), C.c_uint64()
    rc = lib().oracle_brute_count(len(qv), _p(qv), len(qe), _p(qe), len(vl), _p(vl), len(e), _p(e), v1, v2,
                                  int(homo), C.byref(c), C.byref(h))
    if rc != 0:
        raise RuntimeError("oracle_brute_count failed")
    return int(c.value), int(h.value)


def graphflow_orders(q_vlabels, q_edges) -> np.ndarray:
    qv = np.ascontiguousarray(q_vlabels, dtype=np.uint32)
    qe = np.ascontiguousarray(q_edges, dtype=np.uint32).reshape(-1, 3)
    out = np.zeros((len(qe), len(qv)), dtype=np.uint32)
    m = lib().oracle_graphflow_orders(len(qv), _p(qv), len(qe), _p(qe), _p(out))
    if m < 0:
        raise RuntimeError("bad query")
    return out[:m]


def ref_run(query: str | os.PathLike, data: str | os.PathLike, stream: str | os.PathLike, algo: str, *,
            threads: int = 1, max_results: int | None = None, want_hash: bool = False,
            max_updates: int | None = None, time_budget: float | None = None, timeout: float | None = None,
            binary: bool = False, homo: bool = False) -> tuple[np.ndarray, dict]:
    """Runs the reference plugins (oracle/_ref/ref_driver) with sequential semantics.

    Returns per-update rows (pos, neg, latency_ns, hash) and the summary lines.
    """
    if not REF_DRIVER.exists():
        raise RuntimeError(f"reference driver not built: {REF_DRIVER}")
    out_csv = Path(os.environ.get("TMPDIR", "/tmp")) / f"ref_{os.getpid()}_{abs(hash((str(data), algo)))}.csv"
    cmd = [str(REF_DRIVER), "-q", str(query), "-D" if binary else "-d", str(data), "-U" if binary else "-u",
           str(stream), "-a", algo, "-t", str(threads), "--out", str(out_csv)]
    if max_results is not None:
        cmd += ["--max-results", str(max_results)]
    if want_hash:
        cmd += ["--hash"]
    if homo:
        cmd += ["--homo", "1"]
    if max_updates is not None:
        cmd += ["--max-updates", str(max_updates)]
    if time_budget is not None:
        cmd += ["--time-budget", str(time_budget)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"ref_driver failed ({r.returncode}): {r.stderr[-2000:]}")
    rows = list(csv.DictReader(open(out_csv)))
    out_csv.unlink(missing_ok=True)
    dt = np.dtype([("pos", "<u8"), ("neg", "<u8"), ("latency_ns", "<u8"), ("hash", "<u8")])
    arr = np.zeros(len(rows), dtype=dt)
    for i, row in enumerate(rows):
        arr[i] = (int(row["pos"]), int(row["neg"]), int(row["latency_ns"]), int(row["hash"]))
    summary = {}
    for line in r.stdout.splitlines():
        if "updates_per_s=" in line:
            for kv in line.split():
                k, v = kv.split("=")
                summary[k] = float(v)
    return arr, summary
