"""CaLiG-style plugin on the GPU: the `calig` program against the reference
CaLiG's own per-update counts, the parallel_calig plugin against the
reference's counts and the oracle on labelled streams with deletions, and its
lighting filter against the oracle's restatement after whole batches."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import ROOT, calig_cases, golden_cases, load_calig, load_golden
from oracle import pyoracle
from paracosm_b200 import ST_CAPPED, ST_OK, UPDATE_DTYPE, Engine, workload

pytestmark = pytest.mark.gpu

CALIG_BIN = ROOT / "paracosm_b200" / "_bin" / "calig"
UNDERCOUNT_AT = 97  # first update where the reference CaLiG counts fewer matches than exist


def _calig(d, tmp_path, *extra):
    out = tmp_path / "per_update.csv"
    r = subprocess.run([str(CALIG_BIN), "-d", str(d / "data"), "-q", str(d / "query"), "-s", str(d / "stream"),
                        "--out", str(out)] + list(extra), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    rows = np.genfromtxt(out, delimiter=",", names=True, dtype=np.int64)
    return rows, r.stderr


def _duplicates(vl, e, stream) -> np.ndarray:
    """Insertions of an edge present at that point of the stream (a vertex
    removal takes its edges with it)."""
    adj: dict[int, set] = {}
    for a, b, _ in np.asarray(e).reshape(-1, 3).tolist():
        adj.setdefault(a, set()).add(b)
        adj.setdefault(b, set()).add(a)
    dup = np.zeros(len(stream), dtype=bool)
    for i, u in enumerate(stream):
        a, b = int(u["id1"]), int(u["id2"])
        if u["type"] == ord("v"):
            if not u["is_add"]:
                for w in adj.pop(a, set()):
                    adj[w].discard(a)
            continue
        if u["is_add"]:
            dup[i] = b in adj.get(a, ())
            adj.setdefault(a, set()).add(b)
            adj.setdefault(b, set()).add(a)
        else:
            adj.get(a, set()).discard(b)
            adj.get(b, set()).discard(a)
    return dup


@pytest.mark.parametrize("mode", ["batched", "plain"])
@pytest.mark.parametrize("case", [c for c in calig_cases() if c != "calig_undercount"])
def test_calig_program_reproduces_the_reference(case, mode, tmp_path):
    g = load_calig(case)
    rows, err = _calig(g["dir"], tmp_path, "--mode", mode, "--batch", "64")
    assert np.array_equal(rows["pos"].astype(np.uint64), g["exp"]), np.nonzero(rows["pos"] != g["exp"])[0][:8]
    assert f"added matches: {int(g['exp'].sum())}" in err
    assert "deleted matches: 0" in err


def test_calig_program_on_the_undercount_case(tmp_path):
    g = load_calig("calig_undercount")
    rows, _ = _calig(g["dir"], tmp_path)
    k = UNDERCOUNT_AT
    assert np.array_equal(rows["pos"][:k].astype(np.uint64), g["exp"][:k])
    assert rows["pos"][k] > g["exp"][k]
    # without the compatibility rule every insertion is counted exactly
    exact, _ = _calig(g["dir"], tmp_path, "--compat", "0")
    want = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], want_hash=False)
    assert np.array_equal(exact["pos"].astype(np.uint64), want["pos"])


@pytest.mark.parametrize("mode", ["batched", "plain"])
@pytest.mark.parametrize("case", golden_cases())
def test_calig_plugin_counts_on_labelled_streams(case, mode):
    g = load_golden(case)
    cap = g["params"]["max_results"] or 0
    homo = g["params"]["homo"]
    with Engine("parallel_calig", max_results=cap, homo=homo, want_hash=True, mode=mode, max_batch=97) as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        res = eng.run(g["stream"])
    x = g["exp"]
    dup = _duplicates(g["vl"], g["e"], g["stream"])
    pos = np.where(dup, 0, x["symbi_pos"]).astype(np.uint64)
    assert np.array_equal(res["pos"], pos), np.nonzero(res["pos"] != pos)[0][:8]
    assert np.array_equal(res["neg"], x["symbi_neg"])
    ok = (res["status"] == ST_OK) & ~dup
    assert np.array_equal(res["hash"][ok], x["symbi_hash"][ok])
    if cap:
        assert np.array_equal(res["status"] == ST_CAPPED, (pos + x["symbi_neg"]) >= cap)


def test_duplicate_insertion_counts_zero():
    vl = np.array([0, 0, 0], dtype=np.uint32)
    e = np.array([(0, 1, 0), (1, 2, 0)], dtype=np.uint32)
    qv = np.array([0, 0, 0], dtype=np.uint32)
    qe = np.array([(0, 1, 0), (1, 2, 0), (0, 2, 0)], dtype=np.uint32)
    ups = np.zeros(3, dtype=UPDATE_DTYPE)
    ups["type"] = ord("e")
    ups["is_add"] = 1
    ups["id1"], ups["id2"] = [0, 2, 0], [2, 0, 1]
    for algo, want in (("parallel_calig", [6, 0, 0]), ("parallel_symbi", [6, 6, 6])):
        with Engine(algo) as eng:
            eng.set_query(qv, qe)
            eng.load_graph(vl, e)
            eng.build_index()
            assert eng.run(ups)["pos"].tolist() == want, algo


def _same_levels(got, want, n):
    assert np.array_equal(got["d1"][:, :n], want["li0"][:, :n]), np.argwhere(got["d1"][:, :n] != want["li0"][:, :n])[:8]
    assert np.array_equal(got["d2"][:, :n], want["li1"][:, :n]), np.argwhere(got["d2"][:, :n] != want["li1"][:, :n])[:8]
    assert not got["d1"][:, n:].any() and not got["d2"][:, n:].any()


@pytest.mark.parametrize("max_batch", [65536, 7])
@pytest.mark.parametrize("case", golden_cases())
def test_lighting_filter_equals_the_oracle_levels(case, max_batch):
    g = load_golden(case)
    homo = g["params"]["homo"]
    s = g["stream"]
    n = len(g["vl"])
    cuts = [0, len(s) // 3, len(s) // 3 + 1, len(s)]
    with Engine("parallel_calig", homo=homo, max_batch=max_batch) as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        _same_levels(eng.index(), pyoracle.calig_index(g["qv"], g["qe"], g["vl"], g["e"], homo=homo,
                                                       with_lit=False), n)
        for a, b in zip(cuts, cuts[1:]):
            eng.run(s[a:b])
            want = pyoracle.calig_index(g["qv"], g["qe"], g["vl"], g["e"], s[:b], homo=homo, with_lit=False)
            _same_levels(eng.index(), want, n)


@pytest.mark.parametrize("case", calig_cases())
def test_lighting_filter_contains_the_reference_lighting(case):
    g = load_calig(case)
    n = len(g["vl"])
    with Engine("parallel_calig") as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        ix = eng.index()
    _same_levels(ix, pyoracle.calig_index(g["qv"], g["qe"], g["vl"], g["e"], with_lit=False), n)
    assert not (g["lit"] & ~ix["d2"][:, :n]).any()


def test_lighting_filter_after_vertex_updates(gen_dir):
    w = workload.generate("c2", gen_dir / "calig_vx", extra=["--log2-n", "12", "--updates", "1500",
                                                             "--insert-frac", "0.7"])
    qv, qe = w.queries[0]
    n = len(w.vlabels)
    # a vertex removal and a re-insertion in the middle of the stream
    v = int(w.stream["id1"][10])
    extra = np.zeros(2, dtype=UPDATE_DTYPE)
    extra["type"] = ord("v")
    extra["is_add"] = [0, 1]
    extra["id1"] = v
    extra["label"] = w.vlabels[v]
    rest = w.stream[700:]
    rest = rest[(rest["id1"] != v) & (rest["id2"] != v)]  # no edge updates at v once it is removed
    s = np.concatenate([w.stream[:700], extra[:1], rest[:200], extra[1:], rest[200:]])
    with Engine("parallel_calig", max_batch=300) as eng:
        eng.set_query(qv, qe)
        eng.load_graph(w.vlabels, w.edges)
        eng.build_index()
        res = eng.run(s)
        want_ix = pyoracle.calig_index(qv, qe, w.vlabels, w.edges, s)
        _same_levels(eng.index(), want_ix, n)
    want = pyoracle.run(qv, qe, w.vlabels, w.edges, s, want_hash=False)
    ok = (want["status"] == ST_OK) & ~_duplicates(w.vlabels, w.edges, s)
    assert np.array_equal(res["pos"][ok], want["pos"][ok])
    assert np.array_equal(res["neg"][ok], want["neg"][ok])


@pytest.mark.parametrize("max_batch", [65536, 7])
@pytest.mark.parametrize("case", ["mixed_2el", "zipf_8q", "homo"])
def test_newsp_filter_levels_equal_the_oracle(case, max_batch):
    """The NewSP-style plugin keeps the same two levels; its search filters by the first."""
    g = load_golden(case)
    homo = g["params"]["homo"]
    s = g["stream"]
    n = len(g["vl"])
    with Engine("parallel_newsp", homo=homo, max_batch=max_batch, want_hash=True) as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        _same_levels(eng.index(), pyoracle.calig_index(g["qv"], g["qe"], g["vl"], g["e"], homo=homo,
                                                       with_lit=False), n)
        res = eng.run(s)
        _same_levels(eng.index(), pyoracle.calig_index(g["qv"], g["qe"], g["vl"], g["e"], s, homo=homo,
                                                       with_lit=False), n)
    x = g["exp"]
    assert np.array_equal(res["pos"], x["symbi_pos"]) and np.array_equal(res["neg"], x["symbi_neg"])
    ok = res["status"] == ST_OK
    assert np.array_equal(res["hash"][ok], x["symbi_hash"][ok])
