"""Seeded workload generator and file formats (CPU only)."""
from __future__ import annotations

import hashlib

import numpy as np

from paracosm_b200 import workload


def _digest(w: workload.Workload) -> str:
    h = hashlib.sha256()
    for a in (w.vlabels, w.edges, w.stream.view(np.uint8)):
        h.update(np.ascontiguousarray(a).tobytes())
    for qv, qe in w.queries:
        h.update(qv.tobytes()); h.update(qe.tobytes())
    return h.hexdigest()


def test_generator_is_deterministic(gen_dir):
    a = workload.generate("c1", gen_dir / "a", reuse=False)
    b = workload.generate("c1", gen_dir / "b", reuse=False)
    assert _digest(a) == _digest(b)
    c = workload.generate("c1", gen_dir / "c", seed=99, reuse=False)
    assert _digest(a) != _digest(c)


def test_c1_shape(gen_dir):
    w = workload.generate("c1", gen_dir / "c1")
    assert len(w.vlabels) == 1 << 14
    assert len(w.edges) + 6554 == 65536  # 10% held out
    assert len(w.stream) == 2000 and np.all(w.stream["is_add"] == 1)
    qv, qe = w.queries[0]
    assert len(qv) == 6
    assert set(np.unique(w.vlabels)) <= {0, 1, 2, 3}


def test_stream_is_valid_against_the_graph(gen_dir):
    w = workload.generate("c2", gen_dir / "c2s", extra=["--log2-n", "12", "--updates", "3000"])
    cur = {(min(a, b), max(a, b)): l for a, b, l in w.edges}
    for u in w.stream:
        k = (min(int(u["id1"]), int(u["id2"])), max(int(u["id1"]), int(u["id2"])))
        if u["is_add"]:
            assert k not in cur
            cur[k] = int(u["label"])
        else:
            assert cur.pop(k) == int(u["label"])
    frac = float(np.mean(w.stream["is_add"]))
    assert abs(frac - 0.9) < 1e-9


def test_dense_query_meets_its_degree_bound(gen_dir):
    w = workload.generate("c2", gen_dir / "dq", extra=["--log2-n", "12", "--updates", "10", "--query", "8:dense:0:3"])
    qv, qe = w.queries[0]
    assert 2 * len(qe) / len(qv) >= 3


def test_text_and_binary_formats_agree(gen_dir, tmp_path):
    w = workload.generate("c1", gen_dir / "txt", text=True, extra=["--log2-n", "10", "--updates", "50"])
    vl, e = workload.read_graph(w.directory / "data.graph")
    assert np.array_equal(vl, w.vlabels) and np.array_equal(e, w.edges)
    s = workload.read_stream(w.directory / "stream.txt")
    assert np.array_equal(s, w.stream)
    workload.write_stream_text(tmp_path / "s.txt", s)
    assert np.array_equal(workload.read_stream(tmp_path / "s.txt"), s)
