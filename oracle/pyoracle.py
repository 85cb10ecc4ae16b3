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
        _lib.oracle_initial_count.restype = C.c_int
        _lib.oracle_initial_count.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                              C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_int,
                                              C.POINTER(C.c_uint64)]
        _lib.oracle_group_assignments.restype = C.c_uint64
        _lib.oracle_group_assignments.argtypes = [C.c_uint32, C.c_void_p, C.c_int]
        _lib.oracle_calig_index.restype = C.c_int
        _lib.oracle_calig_index.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                            C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_int, C.c_uint64,
                                            C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_index.restype = C.c_int
        _lib.oracle_index.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p,
                                      C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_int,
                                      C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                      C.c_void_p]
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


def initial_count(q_vlabels, q_edges, vlabels, edges, updates=None, *, homo: bool = False) -> int:
    """Embeddings of the query in the graph after the given updates (InitialMatching)."""
    qv = np.ascontiguousarray(q_vlabels, dtype=np.uint32)
    qe = np.ascontiguousarray(q_edges, dtype=np.uint32).reshape(-1, 3)
    vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
    e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 3)
    u = np.ascontiguousarray(updates if updates is not None else np.zeros(0, UPDATE_DTYPE), dtype=UPDATE_DTYPE)
    c = C.c_uint64()
    rc = lib().oracle_initial_count(len(qv), _p(qv), len(qe), _p(qe), len(vl), _p(vl), len(e), _p(e), len(u), _p(u),
                                    int(homo), C.byref(c))
    if rc != 0:
        raise RuntimeError("oracle_initial_count failed")
    return int(c.value)


INDEX_ALGOS = {"turboflux": 1, "symbi": 2, "parallel_turboflux": 1, "parallel_symbi": 2}


def index(q_vlabels, q_edges, vlabels, edges, updates=None, *, algo: str = "symbi") -> dict:
    """Candidate index of the TurboFlux / SymBi plugin after the given updates.

    Returns root, order (serialized tree), parents (sorted lists per query
    vertex) and d1 / d2 as bool arrays of shape [n_qv, n_vertices].
    """
    qv = np.ascontiguousarray(q_vlabels, dtype=np.uint32)
    qe = np.ascontiguousarray(q_edges, dtype=np.uint32).reshape(-1, 3)
    vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
    e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 3)
    u = np.ascontiguousarray(updates if updates is not None else np.zeros(0, UPDATE_DTYPE), dtype=UPDATE_DTYPE)
    nmax = len(vl)
    for r in u:
        if r["type"] == ord("v"):
            nmax = max(nmax, int(r["id1"]) + 1)
    words = (nmax + 63) // 64 + 1
    root = C.c_uint32()
    order = np.zeros(len(qv), dtype=np.uint32)
    parents = np.zeros(len(qv), dtype=np.uint32)
    d1 = np.zeros((len(qv), words), dtype=np.uint64)
    d2 = np.zeros((len(qv), words), dtype=np.uint64)
    n = lib().oracle_index(len(qv), _p(qv), len(qe), _p(qe), len(vl), _p(vl), len(e), _p(e), len(u), _p(u),
                           INDEX_ALGOS[algo], C.byref(root), _p(order), _p(parents), words, _p(d1), _p(d2))
    if n < 0:
        raise RuntimeError(f"oracle_index failed: {n}")
    bits = lambda a: np.unpackbits(a.view(np.uint8), axis=1, bitorder="little")[:, :n].astype(bool)  # noqa: E731
    par = [[p for p in range(len(qv)) if (int(parents[q]) >> p) & 1] for q in range(len(qv))]
    return {"root": int(root.value), "order": order.tolist(), "parents": par, "d1": bits(d1), "d2": bits(d2)}


def group_assignments(g: int, classes: dict, homo: bool = False) -> int:
    """Injective assignments of g same-label tail positions; classes maps a
    membership bitmask M to the number of candidates with exactly that membership."""
    n = np.zeros(8, dtype=np.uint64)
    for m, c in classes.items():
        n[m] = c
    return int(lib().oracle_group_assignments(g, _p(n), int(homo)))


def calig_index(q_vlabels, q_edges, vlabels, edges, updates=None, *, homo: bool = False,
                with_lit: bool = True) -> dict:
    """CaLiG-style flags after the given updates: li0 / li1 (the two levels the
    engine maintains) and lit (the reference CaLiG's lighting after static
    filtering), as bool arrays of shape [n_qv, n_vertices]."""
    qv = np.ascontiguousarray(q_vlabels, dtype=np.uint32)
    qe = np.ascontiguousarray(q_edges, dtype=np.uint32).reshape(-1, 3)
    vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
    e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 3)
    u = np.ascontiguousarray(updates if updates is not None else np.zeros(0, UPDATE_DTYPE), dtype=UPDATE_DTYPE)
    nmax = len(vl)
    for r in u:
        if r["type"] == ord("v"):
            nmax = max(nmax, int(r["id1"]) + 1)
    words = (nmax + 63) // 64 + 1
    li0 = np.zeros((len(qv), words), dtype=np.uint64)
    li1 = np.zeros((len(qv), words), dtype=np.uint64)
    lit = np.zeros((len(qv), words), dtype=np.uint64)
    n = lib().oracle_calig_index(len(qv), _p(qv), len(qe), _p(qe), len(vl), _p(vl), len(e), _p(e), len(u), _p(u),
                                 int(homo), words, _p(li0), _p(li1), _p(lit) if with_lit else 0)
    if n < 0:
        raise RuntimeError(f"oracle_calig_index failed: {n}")
    bits = lambda a: np.unpackbits(a.view(np.uint8), axis=1, bitorder="little")[:, :n].astype(bool)  # noqa: E731
    out = {"li0": bits(li0), "li1": bits(li1)}
    if with_lit:
        out["lit"] = bits(lit)
    return out


def parse_index_dump(text: str, n_vertices: int) -> dict:
    """Parses ref_driver --dump-index output into {at: index dict} (same keys as index())."""
    out: dict = {}
    cur = None
    for line in text.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "at":
            cur = {"parents": {}, "d1": {}, "d2": {}}
            out[int(t[1])] = cur
        elif t[0] == "root":
            cur["root"] = int(t[1])
        elif t[0] == "order":
            cur["order"] = [int(x) for x in t[1:]]
        elif t[0] == "parents":
            cur["parents"][int(t[1])] = sorted(int(x) for x in t[2:])
        elif t[0] in ("d1", "d2"):
            cur[t[0]][int(t[1])] = [int(x) for x in t[2:]]
    for cur in out.values():
        nq = len(cur["order"])
        cur["parents"] = [cur["parents"][q] for q in range(nq)]
        for k in ("d1", "d2"):
            a = np.zeros((nq, n_vertices), dtype=bool)
            for q, vs in cur[k].items():
                a[q, vs] = True
            cur[k] = a
    return out


def ref_index(query, data, stream, algo: str, at: list[int], n_vertices: int, *, timeout: float = 600) -> dict:
    """The reference plugin's own index state after each update count in `at` (0: after preprocessing)."""
    if not REF_DRIVER.exists():
        raise RuntimeError(f"reference driver not built: {REF_DRIVER}")
    tmp = Path(os.environ.get("TMPDIR", "/tmp")) / f"refidx_{os.getpid()}_{algo}.txt"
    cmd = [str(REF_DRIVER), "-q", str(query), "-d", str(data), "-u", str(stream), "-a", algo, "--dump-index",
           str(tmp), "--dump-at", ",".join(str(x) for x in at)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"ref_driver failed ({r.returncode}): {r.stderr[-2000:]}")
    text = tmp.read_text()
    tmp.unlink(missing_ok=True)
    return parse_index_dump(text, n_vertices)


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
