"""CPU checks of the oracle (the CPU restatement) against the reference's own
outputs (golden fixtures) and against exhaustive brute force."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases, load_golden, load_golden_index
from oracle import pyoracle

UPD = pyoracle.UPDATE_DTYPE


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_matches_reference_symbi(case):
    g = load_golden(case)
    p = g["params"]
    r = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], max_results=p["max_results"] or 0,
                     homo=p["homo"])
    exp = g["exp"]
    assert np.array_equal(r["pos"], exp["symbi_pos"])
    assert np.array_equal(r["neg"], exp["symbi_neg"])
    ok = r["status"] == pyoracle.ST_OK
    assert np.array_equal(r["hash"][ok], exp["symbi_hash"][ok])


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_matches_reference_graphflow_and_turboflux_positives(case):
    g = load_golden(case)
    p = g["params"]
    r = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], max_results=p["max_results"] or 0,
                     homo=p["homo"])
    exp = g["exp"]
    # sequential TurboFlux positives are exact; its negatives skip the anchor label
    # check (TurboFlux/turboflux.cpp:975), so they are only compared with one edge label.
    assert np.array_equal(r["pos"], exp["turboflux_pos"])
    if p["max_results"] is None:
        # GraphFlow checks the cap only between seeds (graphflow.cpp:328), so only uncapped runs compare
        assert np.array_equal(r["pos"], exp["graphflow_pos"])
        assert np.array_equal(r["neg"], exp["graphflow_neg"])


def _tiny_case(seed: int, n: int = 9, m: int = 16, nvl: int = 2, nel: int = 2, nq: int = 4, nup: int = 30):
    rng = np.random.default_rng(seed)
    vl = rng.integers(0, nvl, n).astype(np.uint32)
    pairs = set()
    while len(pairs) < m:
        a, b = rng.integers(0, n, 2)
        if a != b:
            pairs.add((min(a, b), max(a, b)))
    pairs = sorted(pairs)
    lab = rng.integers(0, nel, len(pairs))
    edges = np.array([(a, b, l) for (a, b), l in zip(pairs, lab)], dtype=np.uint32)
    # query: random connected graph on nq vertices
    qv = rng.integers(0, nvl, nq).astype(np.uint32)
    qe = [(i, int(rng.integers(0, i)), int(rng.integers(0, nel))) for i in range(1, nq)]
    extra = rng.integers(0, 2)
    for _ in range(extra):
        a, b = sorted(rng.choice(nq, 2, replace=False))
        if not any((x == a and y == b) or (x == b and y == a) for x, y, _ in qe):
            qe.append((int(a), int(b), int(rng.integers(0, nel))))
    qe = np.array(qe, dtype=np.uint32)
    # stream over a random set of pairs, insert if absent else delete
    cur = {(a, b): l for a, b, l in edges}
    ups = np.zeros(nup, dtype=UPD)
    for i in range(nup):
        a, b = rng.integers(0, n, 2)
        while a == b:
            a, b = rng.integers(0, n, 2)
        k = (min(a, b), max(a, b))
        if k in cur and rng.random() < 0.6:
            ups[i] = (ord("e"), 0, 0, a, b, cur[k])
            del cur[k]
        else:
            l = int(rng.integers(0, nel))
            ups[i] = (ord("e"), 1, 0, a, b, l)
            cur.setdefault(k, l)
    return vl, edges, qv, qe, ups


@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("homo", [False, True])
def test_oracle_matches_brute_force(seed, homo):
    vl, edges, qv, qe, ups = _tiny_case(seed)
    r = pyoracle.run(qv, qe, vl, edges, ups, homo=homo)
    cur = {(min(a, b), max(a, b)): l for a, b, l in edges}
    for i, u in enumerate(ups):
        a, b = int(u["id1"]), int(u["id2"])
        k = (min(a, b), max(a, b))
        if u["is_add"]:
            dup = k in cur
            cur.setdefault(k, int(u["label"]))
            if dup and cur[k] != int(u["label"]):
                continue  # duplicate insert with another label: counted with the given label, not the graph's
        elif k not in cur:
            assert r["status"][i] == pyoracle.ST_INVALID and r["neg"][i] == 0
            continue
        el = np.array([(x, y, l) for (x, y), l in sorted(cur.items())], dtype=np.uint32).reshape(-1, 3)
        c, h = pyoracle.brute_count(qv, qe, vl, el, a, b, homo=homo)
        got = r["pos"][i] if u["is_add"] else r["neg"][i]
        assert got == c, (i, got, c)
        assert r["hash"][i] == h
        if not u["is_add"]:
            del cur[k]


def test_oracle_cap_stops_at_exactly_the_cap():
    g = load_golden("capped")
    r = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], max_results=40)
    capped = r["status"] == pyoracle.ST_CAPPED
    assert capped.any()
    assert np.all((r["pos"] + r["neg"])[capped] == 40)
    full = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], max_results=0)
    tot = full["pos"] + full["neg"]
    assert np.array_equal(np.minimum(tot, 40), r["pos"] + r["neg"])
    assert np.array_equal(capped, tot >= 40)


@pytest.mark.parametrize("algo", ["symbi", "turboflux"])
@pytest.mark.parametrize("case", golden_cases())
def test_oracle_index_matches_the_reference_plugins_own_index(case, algo):
    """Root, DAG and the d1 / d2 flags, against the state read out of the reference's
    SymBi / TurboFlux objects after preprocessing, half of the stream and all of it."""
    g = load_golden(case)
    ref = load_golden_index(case, algo)
    for at, r in ref.items():
        o = pyoracle.index(g["qv"], g["qe"], g["vl"], g["e"], g["stream"][:at], algo=algo)
        assert o["root"] == r["root"] and o["order"] == r["order"] and o["parents"] == r["parents"]
        n = r["d1"].shape[1]
        assert np.array_equal(o["d1"][:, :n], r["d1"]), at
        assert np.array_equal(o["d2"][:, :n], r["d2"]), at
        assert not o["d1"][:, n:].any() and not o["d2"][:, n:].any()


def test_oracle_index_is_the_fixpoint_by_definition():
    """d1 / d2 on a tiny graph, checked against a direct evaluation of the definition."""
    rng = np.random.default_rng(5)
    n = 40
    vl = rng.integers(0, 2, n).astype(np.uint32)
    e = np.array([(a, b, int(rng.integers(0, 2))) for a in range(n) for b in range(a + 1, n) if rng.random() < 0.12],
                 dtype=np.uint32)
    qv = np.array([0, 1, 0, 1], dtype=np.uint32)
    qe = np.array([(0, 1, 0), (1, 2, 1), (2, 3, 0), (0, 2, 0)], dtype=np.uint32)
    adj = {}
    for a, b, l in e:
        adj.setdefault(int(a), []).append((int(b), int(l)))
        adj.setdefault(int(b), []).append((int(a), int(l)))
    ql = {(int(a), int(b)): int(l) for a, b, l in qe}
    ql.update({(b, a): l for (a, b), l in ql.items()})
    for algo in ("symbi", "turboflux"):
        o = pyoracle.index(qv, qe, vl, e, algo=algo)
        par = o["parents"]
        chd = [[c for c in range(4) if u in par[c]] for u in range(4)]
        d1 = np.zeros((4, n), bool)
        d2 = np.zeros((4, n), bool)
        sup = lambda v, w_lab, el, flag: any(vl[w] == w_lab and l == el and flag[w] for w, l in adj.get(v, []))  # noqa: E731
        for u in o["order"]:
            for v in range(n):
                d1[u, v] = vl[v] == qv[u] and all(sup(v, qv[p], ql[(u, p)], d1[p]) for p in par[u])
        for u in reversed(o["order"]):
            for v in range(n):
                d2[u, v] = d1[u, v] and all(sup(v, qv[c], ql[(u, c)], d2[c]) for c in chd[u])
        assert np.array_equal(o["d1"], d1) and np.array_equal(o["d2"], d2)
        assert o["order"][0] == o["root"] and par[o["root"]] == []


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_initial_count_matches_the_reference_csm(case):
    """InitialMatching counts printed by the reference's own csm driver (initial.json)."""
    import json
    g = load_golden(case)
    want = json.loads((g["dir"] / "initial.json").read_text())
    got = pyoracle.initial_count(g["qv"], g["qe"], g["vl"], g["e"], homo=g["params"]["homo"])
    assert got == want["graphflow"] == want["symbi"] == want["turboflux"]


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_tail_counting_gives_the_enumeration_counts(case):
    """The counting search (want_hash = 0: the independent tail of each order is
    counted, not enumerated) gives the reference's counts."""
    g = load_golden(case)
    cap = g["params"]["max_results"] or 0
    kw = dict(max_results=cap, homo=g["params"]["homo"])
    full = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], want_hash=True, **kw)
    tail = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], want_hash=False, **kw)
    assert np.array_equal(tail["pos"], full["pos"]) and np.array_equal(tail["neg"], full["neg"])
    assert np.array_equal(tail["status"], full["status"])
    assert np.array_equal(tail["pos"], g["exp"]["symbi_pos"])


# sparse queries over three labels whose orders end in tails with three
# vertices of one label; the second one has capped updates
GROUP3 = [
    (["--avg-degree", "3", "--seed", "3", "--query", "10:sparse:1"], 0),
    (["--avg-degree", "4", "--seed", "1", "--query", "9:sparse:0"], 1_000_000),
]


@pytest.mark.parametrize("spec", range(len(GROUP3)))
def test_oracle_tail_counting_with_groups_of_three(gen_dir, spec):
    from paracosm_b200 import workload
    args, cap = GROUP3[spec]
    w = workload.generate("c2", gen_dir / f"tail3_{spec}", extra=[
        "--log2-n", "11", "--vlabels", "3", "--zipf", "0", "--elabels", "2", "--updates", "300",
        "--insert-frac", "0.8"] + args)
    qv, qe = w.queries[0]
    full = pyoracle.run(qv, qe, w.vlabels, w.edges, w.stream, max_results=cap, want_hash=True)
    tail = pyoracle.run(qv, qe, w.vlabels, w.edges, w.stream, max_results=cap, want_hash=False)
    assert np.array_equal(tail["pos"], full["pos"]) and np.array_equal(tail["neg"], full["neg"])
    assert np.array_equal(tail["status"], full["status"])
    assert full["pos"].sum() > 0


def test_group_assignments_equal_brute_force():
    """The counting search's group count against an explicit enumeration of injective
    (and, under homomorphism, arbitrary) assignments on random candidate sets."""
    import itertools
    rng = np.random.default_rng(7)
    for _ in range(300):
        g = int(rng.integers(1, 4))
        universe = int(rng.integers(1, 9))
        sets = [set(np.nonzero(rng.random(universe) < 0.5)[0].tolist()) for _ in range(g)]
        classes = {}
        for x in range(universe):
            m = sum(1 << i for i in range(g) if x in sets[i])
            if m:
                classes[m] = classes.get(m, 0) + 1
        inj = sum(1 for t in itertools.product(*[sorted(s) for s in sets]) if len(set(t)) == g)
        anyway = int(np.prod([len(s) for s in sets]))
        assert pyoracle.group_assignments(g, classes) == inj, (sets, classes)
        assert pyoracle.group_assignments(g, classes, homo=True) == anyway


def test_oracle_matches_reference_symbi_on_the_c3_shape(tmp_path_factory):
    """The C3 shape (16-vertex dense query, 16 Zipf vertex labels, 4 edge labels) at 2^16
    vertices: the oracle's counts and match-set hashes equal the reference SymBi's on the first
    13,000 updates (six of them nonzero, deletions among them; the rest of the 70,000-update
    stream is checked on the GPU against the same fixture)."""
    from conftest import load_c3_shape
    c = load_c3_shape(tmp_path_factory.mktemp("c3_shape"))
    w, x = c["w"], c["exp"]
    qv, qe = w.queries[0]
    n = 13_000
    ref = pyoracle.run(qv, qe, w.vlabels, w.edges, w.stream[:n], max_results=c["params"]["max_results"])
    assert np.array_equal(ref["pos"], x["pos"][:n])
    assert np.array_equal(ref["neg"], x["neg"][:n])
    assert np.array_equal(ref["hash"], x["hash"][:n])
    assert int(((x["pos"][:n] + x["neg"][:n]) > 0).sum()) == 6


def _selfloop():
    import csv

    from conftest import GOLDEN
    from paracosm_b200 import workload
    d = GOLDEN / "selfloop"
    qv, qe = workload.read_graph(d / "query.graph")
    vl, e = workload.read_graph(d / "data.graph")
    s = workload.read_stream(d / "stream.txt")
    rows = list(csv.DictReader(open(d / "selfloop.csv")))
    x = {k: np.array([int(r[k]) for r in rows], dtype=np.uint64) for k in rows[0] if k != "idx"}
    return qv, qe, vl, e, s, x


def test_self_loops_in_the_data_graph():
    """Data self loops are dropped when a graph is loaded.  Without --homo a loop can never be
    part of an embedding, so the counts equal the reference SymBi's on the graph with its loops.
    Under --homo the reference can map a query edge between two same-label vertices onto a loop
    (its Graph keeps a loop's vertex twice in its own neighbour list); the restatement counts as
    the reference does on the same graph without the loops, and the fixture records where the two
    differ."""
    qv, qe, vl, e, s, x = _selfloop()
    assert int((e[:, 0] == e[:, 1]).sum()) == 80
    r = pyoracle.run(qv, qe, vl, e, s, want_hash=False)
    assert np.array_equal(r["pos"], x["pos"]) and np.array_equal(r["neg"], x["neg"])
    r = pyoracle.run(qv, qe, vl, e, s, homo=True, want_hash=False)
    assert np.array_equal(r["pos"], x["homo_noloop_pos"]) and np.array_equal(r["neg"], x["homo_noloop_neg"])
    differ = (x["homo_pos"] != x["homo_noloop_pos"]) | (x["homo_neg"] != x["homo_noloop_neg"])
    assert int(differ.sum()) == 112
