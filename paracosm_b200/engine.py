"""Python host over the C ABI: an `Engine` object and `matching`-style plugins.

The plugin classes mirror the reference's plugin interface `class matching`
(ParaCOSM/CSM/matching/matching.h:9-66) and constructors
(ParaCOSM/CSM/matching/main.cpp:740-757), so code written against the
reference reads the same:

    q, d = Graph.from_file(qpath), Graph.from_file(dpath)
    mm = Parallel_TurboFlux(q, d, max_num_results, print_prep, print_enum, homo, thread_num, auto_tuning)
    mm.Preprocessing()
    mm.AddEdge(v1, v2, label); mm.RemoveEdge(v1, v2)
    mm.GetNumPositiveResults(); mm.GetNumNegativeResults()

Per-update calls run one update per launch sequence (the plain GPU form);
`Engine.submit` runs whole batches.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import (ALGORITHMS, MODE_BATCHED, MODE_PLAIN, RESULT_DTYPE, UPDATE_DTYPE, CsmCfg, CsmIndexInfo, CsmStats, check,
                   load_library)

NOT_EXIST = 0xFFFFFFFF


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


class Engine:
    """One engine context (one GPU, one standing query)."""

    def __init__(self, algorithm: str | int = "parallel_graphflow", *, max_results: int = 0, homo: bool = False,
                 mode: str = "batched", max_batch: int = 65536, want_hash: bool = False, device: int = 0,
                 deadline_ns: int = 0, hbm_budget_bytes: int = 0, warps_per_block: int = 0,
                 blocks_per_sm: int = 0, turboflux_compat: bool = False, vertex_headroom: int = 0,
                 graphs: bool = False, shard_rank: int = 0, shard_count: int = 1, donate_every: int = 0,
                 split_deep: int = 0, enum_capacity: int = 0, tail_enumerate: bool = False):
        self.lib = load_library()
        cfg = CsmCfg()
        self.lib.csm_gpu_default_cfg(C.byref(cfg))
        cfg.algorithm = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        cfg.homomorphism = int(bool(homo))
        cfg.max_results = int(max_results)
        cfg.deadline_ns = int(deadline_ns)
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.mode = MODE_PLAIN if mode == "plain" else MODE_BATCHED
        cfg.max_batch = int(max_batch)
        cfg.want_hash = int(bool(want_hash))
        cfg.device = int(device)
        cfg.turboflux_compat = int(bool(turboflux_compat))
        cfg.warps_per_block = int(warps_per_block)
        cfg.blocks_per_sm = int(blocks_per_sm)
        cfg.vertex_headroom = int(vertex_headroom)
        cfg.graphs = int(bool(graphs))
        cfg.shard_rank = int(shard_rank)
        cfg.shard_count = int(shard_count)
        cfg.donate_every = int(donate_every)
        cfg.split_deep = int(split_deep)
        cfg.enum_capacity = int(enum_capacity)
        cfg.tail_enumerate = int(bool(tail_enumerate))
        self.cfg = cfg
        h = C.c_void_p()
        check(self.lib, self.lib.csm_gpu_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.submitted = 0
        self.attached: list[Engine] = []
        self.owner: Engine | None = None

    # -- setup ---------------------------------------------------------
    def set_query(self, vlabels, edges) -> None:
        vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
        self._nq = len(vl)
        e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 3)
        check(self.lib, self.lib.csm_gpu_set_query(self.h, len(vl), _ptr(vl), len(e), _ptr(e)))

    def load_graph(self, vlabels, edges) -> None:
        vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
        e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 3)
        check(self.lib, self.lib.csm_gpu_load_graph(self.h, len(vl), _ptr(vl), len(e), _ptr(e)))

    def reserve_labels(self, vlabels=(), elabels=()) -> None:
        """Keeps these labels distinct (for queries attached later); before load_graph."""
        vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
        el = np.ascontiguousarray(elabels, dtype=np.uint32)
        check(self.lib, self.lib.csm_gpu_reserve_labels(self.h, len(vl), _ptr(vl), len(el), _ptr(el)))

    def build_index(self) -> None:
        check(self.lib, self.lib.csm_gpu_build_index(self.h))

    def attach(self, vlabels, edges, algorithm: str | int = "parallel_graphflow", *, max_results: int = 0,
               want_hash: bool = False, warps_per_block: int = 0, blocks_per_sm: int = 0,
               enum_capacity: int = 0, tail_enumerate: bool = False) -> "Engine":
        """A standing query on this engine's graph; its results follow every submit to this engine."""
        cfg = CsmCfg()
        self.lib.csm_gpu_default_cfg(C.byref(cfg))
        cfg.algorithm = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        cfg.max_results = int(max_results)
        cfg.want_hash = int(bool(want_hash))
        cfg.warps_per_block = int(warps_per_block)
        cfg.blocks_per_sm = int(blocks_per_sm)
        cfg.enum_capacity = int(enum_capacity)
        cfg.tail_enumerate = int(bool(tail_enumerate))
        vl = np.ascontiguousarray(vlabels, dtype=np.uint32)
        e = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 3)
        h = C.c_void_p()
        check(self.lib, self.lib.csm_gpu_attach_query(self.h, C.byref(cfg), len(vl), _ptr(vl), len(e), _ptr(e),
                                                      C.byref(h)))
        a = Engine.__new__(Engine)
        a.lib, a.cfg, a.h, a.submitted, a.attached, a.owner = self.lib, cfg, h, self.submitted, [], self
        a._nq = len(vl)
        self.attached.append(a)
        return a

    def initial_match(self) -> int:
        c = C.c_uint64()
        check(self.lib, self.lib.csm_gpu_initial_match(self.h, C.byref(c)))
        return int(c.value)

    def autotune(self, sample: np.ndarray) -> dict:
        """Picks the search launch shape from timings on sample edges (the graph is not modified)."""
        u = np.ascontiguousarray(sample, dtype=UPDATE_DTYPE)
        w, b, de, sd, ms = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_float()
        check(self.lib, self.lib.csm_gpu_autotune(self.h, len(u), _ptr(u), C.byref(w), C.byref(b), C.byref(de),
                                                  C.byref(sd), C.byref(ms)))
        return {"warps_per_block": int(w.value), "blocks_per_sm": int(b.value), "donate_every": int(de.value),
                "split_deep": int(sd.value), "sample_search_ms": float(ms.value)}

    # -- updates -------------------------------------------------------
    def classify(self, updates: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(updates, dtype=UPDATE_DTYPE)
        out = np.zeros(len(u), dtype=np.uint8)
        check(self.lib, self.lib.csm_gpu_classify(self.h, len(u), _ptr(u), _ptr(out)))
        return out

    def submit(self, updates: np.ndarray) -> int:
        """Queues host-memory updates; returns the sequence number of the first."""
        u = updates if (updates.dtype == UPDATE_DTYPE and updates.flags.c_contiguous) else \
            np.ascontiguousarray(updates, dtype=UPDATE_DTYPE)
        first = self.submitted
        check(self.lib, self.lib.csm_gpu_submit(self.h, len(u), _ptr(u)))
        self._advance(len(u))
        return first

    def submit_ptr(self, ptr: int, n: int) -> int:
        """Queues n updates from a raw host pointer (e.g. pinned memory)."""
        first = self.submitted
        check(self.lib, self.lib.csm_gpu_submit(self.h, n, ptr))
        self._advance(n)
        return first

    def submit_device(self, dptr: int, n: int) -> int:
        """Queues n updates already in device memory (e.g. a CUDA tensor's data_ptr())."""
        first = self.submitted
        check(self.lib, self.lib.csm_gpu_submit_device(self.h, n, dptr))
        self._advance(n)
        return first

    def _advance(self, n: int) -> None:
        self.submitted += n
        for a in self.attached:
            a.submitted += n

    def poll(self) -> bool:
        """True when every submitted update has a result (does not block)."""
        d = C.c_int()
        check(self.lib, self.lib.csm_gpu_poll(self.h, C.byref(d)))
        return bool(d.value)

    def wait(self, timeout_ns: int = 0) -> None:
        check(self.lib, self.lib.csm_gpu_wait(self.h, timeout_ns))

    def results(self, first: int, n: int) -> np.ndarray:
        out = np.zeros(n, dtype=RESULT_DTYPE)
        check(self.lib, self.lib.csm_gpu_results(self.h, first, n, _ptr(out)))
        return out

    def results_device(self) -> tuple[int, int]:
        p = C.c_void_p()
        n = C.c_uint64()
        check(self.lib, self.lib.csm_gpu_results_device(self.h, C.byref(p), C.byref(n)))
        return int(p.value or 0), int(n.value)

    def run(self, updates: np.ndarray) -> np.ndarray:
        first = self.submit(updates)
        self.wait()
        return self.results(first, len(updates))

    def stats(self) -> dict:
        s = CsmStats()
        check(self.lib, self.lib.csm_gpu_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in CsmStats._fields_}

    def search_counters(self) -> dict:
        out = np.zeros(10, dtype=np.uint64)
        check(self.lib, self.lib.csm_gpu_search_counters(self.h, _ptr(out), 10))
        names = ["busy_ns", "idle_ns", "iters", "donations", "starved", "checks", "checks_hungry", "root_busy_ns",
                 "last_root_ns", "max_task_ns"]
        return {k: int(v) for k, v in zip(names, out)}

    def index(self, n_vertices: int | None = None) -> dict | None:
        """The TurboFlux / SymBi candidate index: root, order, parents (sorted lists) and d1 / d2
        as bool arrays [n_qv, n_vertices]; None for GraphFlow."""
        info = CsmIndexInfo()
        check(self.lib, self.lib.csm_gpu_index_info(self.h, C.byref(info)))
        if info.algorithm == 0 or info.n_qv == 0:
            return None
        nq, words = int(info.n_qv), int(info.words)
        out = {"root": int(info.root), "order": [int(x) for x in info.order[:nq]],
               "parents": [[p for p in range(nq) if (int(info.parents[u]) >> p) & 1] for u in range(nq)],
               "d1_count": int(info.d1_count), "d2_count": int(info.d2_count)}
        n = n_vertices if n_vertices is not None else 64 * words
        for which, key in ((1, "d1"), (2, "d2")):
            buf = np.zeros((nq, words), dtype=np.uint64)
            check(self.lib, self.lib.csm_gpu_index_flags(self.h, which, _ptr(buf), words))
            out[key] = np.unpackbits(buf.view(np.uint8), axis=1, bitorder="little")[:, :n].astype(bool)
        return out

    def matches(self, max_records: int | None = None) -> tuple[np.ndarray, int]:
        """Embeddings of the last submit as rows (update index within the submit, then the data vertex
        of each query vertex), and the number found (above the capacity when some were dropped)."""
        if not hasattr(self, "_nq"):
            raise RuntimeError("set the query first")
        cap = int(self.cfg.enum_capacity) if max_records is None else int(max_records)
        n, found = C.c_uint64(), C.c_uint64()
        buf = np.zeros((max(cap, 1), 1 + self._nq), dtype=np.uint32)
        check(self.lib, self.lib.csm_gpu_matches(self.h, _ptr(buf), cap, C.byref(n), C.byref(found)))
        return buf[: int(n.value)], int(found.value)

    def stream(self) -> int:
        """cudaStream_t of the engine (for CUDA events on the launching stream)."""
        return int(self.lib.csm_gpu_stream(self.h) or 0)

    def kernel_launches(self) -> int:
        return int(self.lib.csm_gpu_kernel_launches(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            if self.owner is not None and self in self.owner.attached:
                self.owner.attached.remove(self)
            self.lib.csm_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------------------
# Graph container with the reference's loaders (ParaCOSM/CSM/graph/graph.cpp:217-285)


@dataclass
class Graph:
    vlabels: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    edges: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.uint32))
    updates: np.ndarray = field(default_factory=lambda: np.zeros(0, UPDATE_DTYPE))

    @staticmethod
    def from_file(path: str) -> "Graph":
        from .workload import read_graph
        vl, e = read_graph(path)
        return Graph(vl, e)

    def LoadUpdateStream(self, path: str) -> None:
        from .workload import read_stream
        self.updates = read_stream(path)

    def NumVertices(self) -> int:
        return len(self.vlabels)

    def NumEdges(self) -> int:
        return len(self.edges)


class matching:
    """Mirror of the reference plugin base class (matching.h:9-66) over the engine."""

    ALGO = "parallel_graphflow"

    def __init__(self, query_graph: Graph, data_graph: Graph, max_num_results: int = 0xFFFFFFFF,
                 print_prep: bool = True, print_enum: bool = False, homo: bool = False, *args, **engine_kw):
        self.query_ = query_graph
        self.data_ = data_graph
        cap = 0 if max_num_results >= 0xFFFFFFFF else int(max_num_results)
        engine_kw.setdefault("mode", "plain")
        self.engine = Engine(self.ALGO, max_results=cap, homo=homo, want_hash=print_enum, **engine_kw)
        self.num_initial_results_ = 0
        self.num_positive_results_ = 0
        self.num_negative_results_ = 0
        self.last_result = None
        self._one = np.zeros(1, dtype=UPDATE_DTYPE)

    def Preprocessing(self) -> None:
        self.engine.set_query(self.query_.vlabels, self.query_.edges)
        self.engine.load_graph(self.data_.vlabels, self.data_.edges)
        self.engine.build_index()

    def InitialMatching(self) -> None:
        self.num_initial_results_ = self.engine.initial_match()

    def _apply(self, t: str, add: int, a: int, b: int, label: int) -> None:
        u = self._one
        u["type"] = ord(t)
        u["is_add"] = add
        u["id1"], u["id2"], u["label"] = a, b, label
        r = self.engine.run(u)[0]
        self.last_result = r
        self.num_positive_results_ += int(r["pos"])
        self.num_negative_results_ += int(r["neg"])

    def AddEdge(self, v1: int, v2: int, label: int) -> None:
        self._apply("e", 1, v1, v2, label)

    def RemoveEdge(self, v1: int, v2: int) -> None:
        self._apply("e", 0, v1, v2, 0)

    def AddVertex(self, vid: int, label: int) -> None:
        self._apply("v", 1, vid, 0, label)

    def RemoveVertex(self, vid: int) -> None:
        self._apply("v", 0, vid, 0, 0)

    def Classify(self, v1: int, v2: int, label: int) -> bool:
        u = self._one.copy()
        u["type"] = ord("e")
        u["is_add"] = 1
        u["id1"], u["id2"], u["label"] = v1, v2, label
        return bool(self.engine.classify(u)[0])

    def GetMemoryCost(self) -> tuple[int, int]:
        s = self.engine.stats()
        return s["index_entries"], s["index_vertices"]

    def GetNumInitialResults(self) -> int:
        return self.num_initial_results_

    def GetNumPositiveResults(self) -> int:
        return self.num_positive_results_

    def GetNumNegativeResults(self) -> int:
        return self.num_negative_results_


class Graphflow(matching):
    ALGO = "graphflow"


class TurboFlux(matching):
    ALGO = "turboflux"


class SymBi(matching):
    ALGO = "symbi"


class _ParallelMixin:
    def __init__(self, query_graph, data_graph, max_num_results=0xFFFFFFFF, print_prep=True, print_enum=False,
                 homo=False, *rest, **engine_kw):
        # thread_num / auto_tuning (main.cpp:747-751) select CPU threads in the
        # reference; the engine sizes its launches itself, so they are accepted and ignored.
        super().__init__(query_graph, data_graph, max_num_results, print_prep, print_enum, homo, **engine_kw)


class Parallel_Graphflow(_ParallelMixin, Graphflow):
    ALGO = "parallel_graphflow"


class Parallel_TurboFlux(_ParallelMixin, TurboFlux):
    ALGO = "parallel_turboflux"


class Parrllel_SymBi(_ParallelMixin, SymBi):
    """Named as the reference's class (ParaCOSM/CSM/matching/Parallel_SymBi/parallel.h:16)."""
    ALGO = "parallel_symbi"


class Parallel_CaLiG(_ParallelMixin, matching):
    """CaLiG's candidate-lighting plugin (ParaCOSM/CSM/matching/Parallel_CaLiG/parallel_calig.cpp), which the
    reference ships as its own program.  An insertion of a present edge counts 0."""
    ALGO = "parallel_calig"


class CSMPP(_ParallelMixin, matching):
    """NewSP's plugin class (ParaCOSM/CSM/matching/Parallel_NewSP/matching/CSMPP.h:8-183): neighbour-label-frequency
    filter; leaf vertices counted together when only counts are wanted."""
    ALGO = "parallel_newsp"


PLUGINS = {
    "graphflow": Graphflow,
    "turboflux": TurboFlux,
    "symbi": SymBi,
    "parallel_graphflow": Parallel_Graphflow,
    "parallel_turboflux": Parallel_TurboFlux,
    "parallel_symbi": Parrllel_SymBi,
    "parallel_calig": Parallel_CaLiG,
    "calig": Parallel_CaLiG,
    "parallel_newsp": CSMPP,
    "newsp": CSMPP,
}
