"""GPU parity: the engine's per-update counts and match-set hashes, through the
C ABI, against the reference's own outputs (golden fixtures) and the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle import pyoracle
from paracosm_b200 import ST_CAPPED, ST_INVALID, ST_OK, ST_TIMED_OUT, UPDATE_DTYPE, Engine, workload

pytestmark = pytest.mark.gpu

ALGOS = ["parallel_graphflow", "parallel_turboflux", "parallel_symbi", "parallel_newsp"]


def run_engine(qv, qe, vl, e, stream, algo="parallel_graphflow", **kw):
    kw.setdefault("want_hash", True)
    with Engine(algo, **kw) as eng:
        eng.set_query(qv, qe)
        eng.load_graph(vl, e)
        eng.build_index()
        res = eng.run(stream)
        stats = eng.stats()
    return res, stats


def assert_same(res, pos, neg, hsh=None, cap=0):
    assert np.array_equal(res["pos"], pos), np.nonzero(res["pos"] != pos)[0][:10]
    assert np.array_equal(res["neg"], neg), np.nonzero(res["neg"] != neg)[0][:10]
    if cap:
        capped = (pos + neg) >= cap
        assert np.array_equal(res["status"] == ST_CAPPED, capped)
    if hsh is not None:
        ok = res["status"] == ST_OK
        assert np.array_equal(res["hash"][ok], hsh[ok])


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("case", golden_cases())
def test_golden_batched(case, algo):
    g = load_golden(case)
    cap = g["params"]["max_results"] or 0
    res, _ = run_engine(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], algo, max_results=cap,
                        homo=g["params"]["homo"])
    x = g["exp"]
    assert_same(res, x["symbi_pos"], x["symbi_neg"], x["symbi_hash"], cap)


@pytest.mark.parametrize("graphs", [False, True])
@pytest.mark.parametrize("case", golden_cases())
def test_golden_plain_one_update_per_launch(case, graphs):
    g = load_golden(case)
    cap = g["params"]["max_results"] or 0
    res, stats = run_engine(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], max_results=cap, mode="plain",
                            homo=g["params"]["homo"], graphs=graphs)
    x = g["exp"]
    assert_same(res, x["symbi_pos"], x["symbi_neg"], x["symbi_hash"], cap)
    assert stats["batches"] == np.sum(g["stream"]["type"] == ord("e"))


@pytest.mark.parametrize("graphs", [False, True])
@pytest.mark.parametrize("max_batch", [2, 7, 64, 333])
def test_batch_boundaries_do_not_change_results(max_batch, graphs):
    g = load_golden("mixed_2el")
    res, _ = run_engine(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], max_batch=max_batch, graphs=graphs,
                        algo="parallel_symbi")
    x = g["exp"]
    assert_same(res, x["symbi_pos"], x["symbi_neg"], x["symbi_hash"])


def test_config1_against_oracle(gen_dir):
    w = workload.generate("c1", gen_dir / "c1")
    qv, qe = w.queries[0]
    ref = pyoracle.run(qv, qe, w.vlabels, w.edges, w.stream)
    res, _ = run_engine(qv, qe, w.vlabels, w.edges, w.stream)
    assert_same(res, ref["pos"], ref["neg"], ref["hash"])
    assert np.array_equal(res["safe"], ref["safe"])


def test_capped_sample_against_oracle(gen_dir):
    w = workload.generate("c2", gen_dir / "c2cap", extra=["--log2-n", "15", "--updates", "1500"])
    qv, qe = w.queries[0]
    cap = 5000
    ref = pyoracle.run(qv, qe, w.vlabels, w.edges, w.stream, max_results=cap)
    for algo in ALGOS:
        res, _ = run_engine(qv, qe, w.vlabels, w.edges, w.stream, algo, max_results=cap)
        assert_same(res, ref["pos"], ref["neg"], ref["hash"], cap)


def _toggle_stream():
    # a small dense graph where one edge is inserted, deleted, re-inserted with
    # another label, duplicated and deleted again inside one batch
    n = 8
    vl = np.zeros(n, dtype=np.uint32)
    edges = np.array([(a, b, 0) for a in range(n) for b in range(a + 1, n) if (a + b) % 3 != 0], dtype=np.uint32)
    qv = np.zeros(4, dtype=np.uint32)
    qe = np.array([(0, 1, 0), (1, 2, 0), (2, 3, 0), (3, 0, 0), (0, 2, 0)], dtype=np.uint32)
    e = lambda add, a, b, l: (ord("e"), add, 0, a, b, l)  # noqa: E731
    ups = [e(1, 0, 3, 0), e(0, 0, 3, 0), e(1, 3, 0, 1), e(1, 0, 3, 0), e(0, 3, 0, 1), e(0, 0, 3, 0),
           e(1, 0, 3, 0), e(0, 1, 2, 0), e(1, 1, 2, 0), e(0, 5, 6, 0), e(0, 5, 6, 0), e(1, 2, 4, 1),
           e(0, 2, 4, 0), e(1, 0, 6, 0), e(0, 0, 6, 0), e(1, 0, 6, 0)]
    return vl, edges, qv, qe, np.array(ups, dtype=UPDATE_DTYPE)


@pytest.mark.parametrize("max_batch", [1, 3, 65536])
def test_same_edge_touched_many_times_in_one_batch(max_batch):
    vl, edges, qv, qe, ups = _toggle_stream()
    ref = pyoracle.run(qv, qe, vl, edges, ups)
    res, _ = run_engine(qv, qe, vl, edges, ups, max_batch=max_batch)
    assert_same(res, ref["pos"], ref["neg"], ref["hash"])
    assert np.array_equal(res["status"] == ST_INVALID, ref["status"] == pyoracle.ST_INVALID)


def test_insert_then_delete_gives_equal_positive_and_negative(gen_dir):
    w = workload.generate("c1", gen_dir / "c1sym", extra=["--log2-n", "12", "--updates", "400"])
    qv, qe = w.queries[0]
    ins = w.stream
    dels = ins[::-1].copy()
    dels["is_add"] = 0
    res, _ = run_engine(qv, qe, w.vlabels, w.edges, np.concatenate([ins, dels]))
    assert np.array_equal(res["pos"][: len(ins)], res["neg"][len(ins):][::-1])
    assert np.array_equal(res["hash"][: len(ins)], res["hash"][len(ins):][::-1])


def test_graph_replay_counts_launches_and_survives_vertex_updates():
    vl = np.array([0, 1, 0, 1, 0, 1], dtype=np.uint32)
    edges = np.array([(0, 1, 0), (1, 2, 0), (2, 3, 0), (3, 4, 0)], dtype=np.uint32)
    qv = np.array([0, 1, 0], dtype=np.uint32)
    qe = np.array([(0, 1, 0), (1, 2, 0)], dtype=np.uint32)
    e = lambda a, b: (ord("e"), 1, 0, a, b, 0)  # noqa: E731
    ups = np.array([e(4, 5), e(0, 5), (ord("v"), 1, 0, 6, 0, 0), e(6, 1), e(6, 3), e(2, 5)], dtype=UPDATE_DTYPE)
    ref = pyoracle.run(qv, qe, vl, edges, ups)
    for mode in ("plain", "batched"):
        with Engine("parallel_symbi", mode=mode, max_batch=2, graphs=True, want_hash=True) as eng:
            eng.set_query(qv, qe)
            eng.load_graph(vl, edges)
            eng.build_index()
            l0 = eng.kernel_launches()
            res = eng.run(ups)
            assert eng.kernel_launches() > l0
        assert_same(res, ref["pos"], ref["neg"], ref["hash"])


def test_vertex_insertion_then_edges():
    vl = np.array([0, 1, 0, 1], dtype=np.uint32)
    edges = np.array([(0, 1, 0), (1, 2, 0), (2, 3, 0)], dtype=np.uint32)
    qv = np.array([0, 1, 0], dtype=np.uint32)
    qe = np.array([(0, 1, 0), (1, 2, 0)], dtype=np.uint32)
    ups = np.array([(ord("v"), 1, 0, 4, 0, 0), (ord("e"), 1, 0, 4, 1, 0), (ord("e"), 1, 0, 4, 3, 0)],
                   dtype=UPDATE_DTYPE)
    ref = pyoracle.run(qv, qe, vl, edges, ups)
    res, _ = run_engine(qv, qe, vl, edges, ups)
    assert_same(res, ref["pos"], ref["neg"], ref["hash"])
    assert res["pos"][1] > 0


def test_vertex_deletion_drops_incident_edges_everywhere():
    """Vertex deletion (the oracle restates Graph::RemoveVertex with the incident edges
    removed from both endpoints): later updates see the vertex gone, and a re-added
    vertex starts without edges."""
    g = load_golden("dense_del")
    s = g["stream"]
    hub = int(np.bincount(g["e"][:, :2].ravel()).argmax())
    vdel = np.array([(ord("v"), 0, 0, hub, 0, 0)], dtype=UPDATE_DTYPE)
    vadd = np.array([(ord("v"), 1, 0, hub, 0, int(g["vl"][hub]))], dtype=UPDATE_DTYPE)
    # while the slot has no label the engine refuses edges that touch it (INVALID); the
    # reference would link them to the unlabeled slot, so the test leaves them out
    mid = s[100:200]
    mid = mid[(mid["id1"] != hub) & (mid["id2"] != hub)]
    ups = np.concatenate([s[:100], vdel, mid, vadd, s[200:]])
    ref = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], ups)
    for algo in ALGOS:
        for mode in ("batched", "plain"):
            res, _ = run_engine(g["qv"], g["qe"], g["vl"], g["e"], ups, algo, mode=mode)
            assert_same(res, ref["pos"], ref["neg"], ref["hash"])
            assert np.array_equal(res["status"] == ST_INVALID, ref["status"] == pyoracle.ST_INVALID)
    with Engine("parallel_symbi") as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        eng.run(ups)
        ix = eng.index(len(g["vl"]))
        want = pyoracle.index(g["qv"], g["qe"], g["vl"], g["e"], ups, algo="symbi")
        assert np.array_equal(ix["d1"][:, :len(g["vl"])], want["d1"][:, :len(g["vl"])])
        assert np.array_equal(ix["d2"][:, :len(g["vl"])], want["d2"][:, :len(g["vl"])])
        assert eng.initial_match() == pyoracle.initial_count(g["qv"], g["qe"], g["vl"], g["e"], ups)


@pytest.mark.parametrize("case", ["c1_small", "mixed_2el", "dense_del", "zipf_8q"])
def test_work_bytes_follow_the_canonical_model(case):
    """GraphFlow without a cap expands exactly the oracle's search-tree nodes, so the
    per-update algorithmic bytes are equal."""
    g = load_golden(case)
    ref = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], homo=g["params"]["homo"])
    res, _ = run_engine(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], "parallel_graphflow",
                        homo=g["params"]["homo"])
    assert np.array_equal(res["work_bytes"], ref["bytes"]), np.nonzero(res["work_bytes"] != ref["bytes"])[0][:10]


def test_deadline_reports_timed_out_with_lower_bounds():
    g = load_golden("capped")  # dense enough that every matching update runs many iterations
    ref = pyoracle.run(g["qv"], g["qe"], g["vl"], g["e"], g["stream"])
    res, _ = run_engine(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], "parallel_symbi", deadline_ns=1)
    timed = res["status"] == ST_TIMED_OUT
    assert timed.any()
    assert np.all(res["pos"][timed] <= ref["pos"][timed]) and np.all(res["neg"][timed] <= ref["neg"][timed])
    ok = res["status"] == ST_OK
    assert np.array_equal(res["pos"][ok], ref["pos"][ok]) and np.array_equal(res["neg"][ok], ref["neg"][ok])
    # a generous deadline changes nothing
    res2, _ = run_engine(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], "parallel_symbi", deadline_ns=60 * 10**9)
    assert_same(res2, ref["pos"], ref["neg"], ref["hash"])


def test_turboflux_compat_needs_the_plain_turboflux_form():
    from paracosm_b200._abi import CSM_EUNSUPPORTED, CsmError
    for kw in ({"algorithm": "parallel_turboflux"}, {"algorithm": "parallel_symbi", "mode": "plain"}):
        with pytest.raises(CsmError) as e:
            Engine(turboflux_compat=True, **kw)
        assert e.value.code == CSM_EUNSUPPORTED


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("case", ["c1_small", "mixed_2el", "dense_del", "zipf_8q"])
def test_match_sets_rebuild_the_reference_hash(case, algo):
    """The embeddings the engine emits (the reference's --print-enum output) are, per update,
    exactly the counted ones: their number is the update's count and their canonical hash is
    sequential SymBi's (golden)."""
    g = load_golden(case)
    x = g["exp"]
    with Engine(algo, enum_capacity=1 << 22, max_batch=97) as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        res = eng.run(g["stream"])
        rec, found = eng.matches()
    total = int((x["symbi_pos"] + x["symbi_neg"]).sum())
    assert found == total == len(rec)
    assert np.array_equal(res["pos"], x["symbi_pos"]) and np.array_equal(res["neg"], x["symbi_neg"])
    n_q = len(g["qv"])
    per = np.bincount(rec[:, 0], minlength=len(g["stream"]))
    assert np.array_equal(per, (x["symbi_pos"] + x["symbi_neg"]).astype(np.int64))
    # the canonical per-update hash, recomputed on the host from the emitted embeddings
    def mix64(z):
        z = z ^ (z >> np.uint64(33)); z = z * np.uint64(0xff51afd7ed558ccd)
        z = z ^ (z >> np.uint64(33)); z = z * np.uint64(0xc4ceb9fe1a85ec53)
        return z ^ (z >> np.uint64(33))
    with np.errstate(over="ignore"):
        s = np.zeros(len(rec), dtype=np.uint64)
        for q in range(n_q):
            s += mix64((np.uint64(q + 1) << np.uint64(32)) ^ rec[:, 1 + q].astype(np.uint64) ^
                       np.uint64(0x9E3779B97F4A7C15))
        h = np.zeros(len(g["stream"]), dtype=np.uint64)
        np.add.at(h, rec[:, 0], mix64(s))
    assert np.array_equal(h, x["symbi_hash"]), np.nonzero(h != x["symbi_hash"])[0][:10]


@pytest.mark.parametrize("case", golden_cases())
def test_turboflux_compat_reproduces_the_reference_turboflux(case):
    """With turboflux_compat (one update per launch), positives, negatives and hashes equal the
    reference's sequential TurboFlux, whose deletions ignore the anchor edge's label."""
    g = load_golden(case)
    cap = g["params"]["max_results"] or 0
    res, _ = run_engine(g["qv"], g["qe"], g["vl"], g["e"], g["stream"], "parallel_turboflux", mode="plain",
                        max_results=cap, homo=g["params"]["homo"], turboflux_compat=True)
    x = g["exp"]
    assert_same(res, x["turboflux_pos"], x["turboflux_neg"], x["turboflux_hash"], cap)


def test_poll_reports_completion_without_blocking():
    import time
    g = load_golden("zipf_8q")
    with Engine("parallel_symbi", want_hash=True) as eng:
        eng.set_query(g["qv"], g["qe"])
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        first = eng.submit(g["stream"])
        t0 = time.time()
        while not eng.poll():
            assert time.time() - t0 < 60
            time.sleep(0.001)
        res = eng.results(first, len(g["stream"]))
    x = g["exp"]
    assert_same(res, x["symbi_pos"], x["symbi_neg"], x["symbi_hash"])


@pytest.mark.parametrize("algo", ["parallel_graphflow", "parallel_symbi", "parallel_turboflux", "parallel_calig"])
def test_plain_form_launches_per_update(algo):
    """One update per launch sequence: an update whose label triple matches no query edge costs at
    most 3 kernel launches (resolve, compaction copy for an insertion, row mutation), any other at
    most 10 (its index round is one cooperative launch); each submit adds one launch that stamps
    its start time.  Counts stay those of the reference."""
    g = load_golden("mixed_2el")
    qv, qe = g["qv"], g["qe"]
    trip, pair = set(), set()
    for a, b, l in qe:
        trip |= {(qv[a], qv[b], l), (qv[b], qv[a], l)}
        pair |= {(qv[a], qv[b]), (qv[b], qv[a])}
    x = g["exp"]
    with Engine(algo, mode="plain") as eng:
        eng.set_query(qv, qe)
        eng.load_graph(g["vl"], g["e"])
        eng.build_index()
        seen = {True: 0, False: 0}
        for i, u in enumerate(g["stream"]):
            l0 = eng.kernel_launches()
            r = eng.run(g["stream"][i:i + 1])[0]
            launches = eng.kernel_launches() - l0
            l1, l2 = g["vl"][u["id1"]], g["vl"][u["id2"]]
            may = (l1, l2, u["label"]) in trip if u["is_add"] else (l1, l2) in pair
            assert launches <= (10 if may else 3) + 1, (i, launches, may)  # + the submit's time stamp
            seen[may] += 1
            if algo != "parallel_calig":
                assert (int(r["pos"]), int(r["neg"])) == (int(x["symbi_pos"][i]), int(x["symbi_neg"][i])), i
        assert seen[True] > 20 and seen[False] > 20


@pytest.mark.parametrize("homo", [False, True])
@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_self_loops_in_the_data_graph(homo, mode):
    """The engine drops data self loops at load: without --homo its counts equal the reference
    SymBi's on the graph with loops, with --homo the reference's on the same graph without them
    (the reference's --homo counts with loops differ; see the self-loop fixture)."""
    import csv

    from conftest import GOLDEN
    d = GOLDEN / "selfloop"
    qv, qe = workload.read_graph(d / "query.graph")
    vl, e = workload.read_graph(d / "data.graph")
    s = workload.read_stream(d / "stream.txt")
    rows = list(csv.DictReader(open(d / "selfloop.csv")))
    x = {k: np.array([int(r[k]) for r in rows], dtype=np.uint64) for k in rows[0] if k != "idx"}
    res, _ = run_engine(qv, qe, vl, e, s, "parallel_symbi", homo=homo, mode=mode, want_hash=False)
    pos, neg = (x["homo_noloop_pos"], x["homo_noloop_neg"]) if homo else (x["pos"], x["neg"])
    assert_same(res, pos, neg)
