"""Workload files: the reference's text formats and the generator's binary containers.

Text formats follow Graph::LoadFromFile / Graph::LoadUpdateStream
(ParaCOSM/CSM/graph/graph.cpp:217-285); binary containers are written by
the seeded generator `paracosm_b200/_bin/csm_gen` (paracosm_b200/host/workload.cpp).
"""
from __future__ import annotations

import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from ._abi import UPDATE_DTYPE

PKG = Path(__file__).resolve().parent
GEN = PKG / "_bin" / "csm_gen"
NOT_EXIST = 0xFFFFFFFF


def read_graph(path: str | os.PathLike) -> tuple[np.ndarray, np.ndarray]:
    """(vertex labels, (m, 3) edge triples) of a text or CSMG graph file."""
    p = Path(path)
    with open(p, "rb") as f:
        head = f.read(4)
    if head == b"CSMG":
        raw = np.fromfile(p, dtype=np.uint8)
        n = int(raw[8:12].view("<u4")[0])
        m = int(raw[12:20].view("<u8")[0])
        vl = raw[28:28 + 4 * n].view("<u4").copy()
        e = raw[28 + 4 * n:28 + 4 * n + 12 * m].view("<u4").reshape(m, 3).copy()
        return vl, e
    vl: list[int] = []
    edges: list[tuple[int, int, int]] = []
    toks = p.read_text().split()
    i = 0
    while i < len(toks):
        t = toks[i]
        if t.startswith("t"):
            i += 3
            continue
        if t == "v":
            vid, lab = int(toks[i + 1]), int(toks[i + 2])
            if vid >= len(vl):
                vl.extend([NOT_EXIST] * (vid + 1 - len(vl)))
            if vl[vid] == NOT_EXIST:
                vl[vid] = lab
            i += 3
            continue
        edges.append((int(toks[i + 1]), int(toks[i + 2]), int(toks[i + 3])))
        i += 4
    return np.array(vl, dtype=np.uint32), np.array(edges, dtype=np.uint32).reshape(-1, 3)


def read_stream(path: str | os.PathLike) -> np.ndarray:
    """Update records (UPDATE_DTYPE) of a text or CSMU stream file."""
    p = Path(path)
    with open(p, "rb") as f:
        head = f.read(4)
    if head == b"CSMU":
        raw = np.fromfile(p, dtype=np.uint8)
        n = int(raw[8:16].view("<u8")[0])
        rec = raw[16:16 + 16 * n].view("<u4").reshape(n, 4)
        out = np.zeros(n, dtype=UPDATE_DTYPE)
        out["type"] = rec[:, 0] & 0xFF
        out["is_add"] = (rec[:, 0] >> 8) & 0xFF
        out["id1"], out["id2"], out["label"] = rec[:, 1], rec[:, 2], rec[:, 3]
        return out
    toks = p.read_text().split()
    recs = []
    i = 0
    while i < len(toks):
        t = toks[i]
        if t in ("v", "-v"):
            recs.append((ord("v"), 1 if t == "v" else 0, 0, int(toks[i + 1]), 0, int(toks[i + 2])))
            i += 3
        else:
            recs.append((ord("e"), 1 if t == "e" else 0, 0, int(toks[i + 1]), int(toks[i + 2]), int(toks[i + 3])))
            i += 4
    return np.array(recs, dtype=UPDATE_DTYPE)


def read_calig_graph(path: str | os.PathLike) -> tuple[np.ndarray, np.ndarray]:
    """(vertex labels, (m, 3) edge triples with label 0) of a graph or query in the
    reference CaLiG program's format (`v id label`, `e a b`;
    ParaCOSM/CSM/matching/CaLiG/README.md).  As its inputQ / inputG
    (ParaCOSM/CSM/matching/Parallel_CaLiG/parallel_calig.cpp:101-143, 271-335):
    a label of -1 reads as 0, and edges with an endpoint beyond the largest
    vertex id are dropped.  Duplicate edges are kept once."""
    toks = Path(path).read_text().split()
    vl: list[int] = []
    raw: list[tuple[int, int]] = []
    i = 0
    while i < len(toks):
        if toks[i] == "v":
            vid, lab = int(toks[i + 1]), int(toks[i + 2])
            if vid >= len(vl):
                vl.extend([NOT_EXIST] * (vid + 1 - len(vl)))
            vl[vid] = max(lab, 0)
        elif toks[i] == "e":
            raw.append((int(toks[i + 1]), int(toks[i + 2])))
        else:
            raise ValueError(f"unexpected token {toks[i]!r} in {path}")
        i += 3
    seen, edges = set(), []
    for a, b in raw:
        if a < 0 or b < 0 or a >= len(vl) or b >= len(vl) or a == b:
            continue
        k = (min(a, b), max(a, b))
        if k not in seen:
            seen.add(k)
            edges.append((a, b, 0))
    return np.array(vl, dtype=np.uint32), np.array(edges, dtype=np.uint32).reshape(-1, 3)


def read_calig_stream(path: str | os.PathLike) -> np.ndarray:
    """Update records of a CaLiG stream: `e a b` inserts (a, b), `e -a-1 -b-1` deletes it."""
    toks = Path(path).read_text().split()
    recs = []
    for i in range(0, len(toks) - 2, 3):
        a, b = int(toks[i + 1]), int(toks[i + 2])
        if a < 0 and b < 0:
            recs.append((ord("e"), 0, 0, -a - 1, -b - 1, 0))
        elif a >= 0 and b >= 0:
            recs.append((ord("e"), 1, 0, a, b, 0))
        else:
            raise ValueError(f"mixed-sign edge record in {path}")
    return np.array(recs, dtype=UPDATE_DTYPE)


def write_graph_text(path: str | os.PathLike, vlabels: np.ndarray, edges: np.ndarray) -> None:
    with open(path, "w") as f:
        for v, l in enumerate(vlabels):
            if l != NOT_EXIST:
                f.write(f"v {v} {l}\n")
        for a, b, l in np.asarray(edges).reshape(-1, 3):
            f.write(f"e {a} {b} {l}\n")


def write_stream_text(path: str | os.PathLike, ups: np.ndarray) -> None:
    with open(path, "w") as f:
        for u in ups:
            if u["type"] == ord("v"):
                f.write(f"{'v' if u['is_add'] else '-v'} {u['id1']} {u['label']}\n")
            else:
                f.write(f"{'e' if u['is_add'] else '-e'} {u['id1']} {u['id2']} {u['label']}\n")


@dataclass
class Workload:
    directory: Path
    vlabels: np.ndarray
    edges: np.ndarray
    stream: np.ndarray
    queries: list  # [(vlabels, edges)]
    meta: dict

    def query_path(self, i: int = 0) -> Path:
        return self.directory / f"query_{i}.graph"


def generate(preset: str, out_dir: str | os.PathLike, *, seed: int | None = None, updates: int | None = None,
             extra: list[str] | None = None, text: bool = False, reuse: bool = True) -> Workload:
    """Runs the seeded generator (csm_gen) and loads the result."""
    out = Path(out_dir)
    if not GEN.exists():
        raise RuntimeError(f"generator missing: {GEN} (run `python -m paracosm_b200.build`)")
    args = [str(GEN), "--preset", preset, "--out", str(out)]
    if seed is not None:
        args += ["--seed", str(seed)]
    if updates is not None:
        args += ["--updates", str(updates)]
    if text:
        args += ["--text"]
    args += list(extra or [])
    stamp = out / "args.txt"
    if not (reuse and stamp.exists() and stamp.read_text() == " ".join(args[1:]) and (out / "data.bin").exists()):
        out.mkdir(parents=True, exist_ok=True)
        subprocess.run(args, check=True, capture_output=True)
        stamp.write_text(" ".join(args[1:]))
    return load(out)


def load(directory: str | os.PathLike) -> Workload:
    d = Path(directory)
    vl, e = read_graph(d / "data.bin")
    s = read_stream(d / "stream.bin")
    qs = []
    i = 0
    while (d / f"query_{i}.graph").exists():
        qs.append(read_graph(d / f"query_{i}.graph"))
        i += 1
    meta = {}
    if (d / "meta.txt").exists():
        for line in (d / "meta.txt").read_text().splitlines():
            if "=" in line:
                k, v = line.split("=", 1)
                meta[k] = v
    return Workload(d, vl, e, s, qs, meta)
