"""ctypes binding of the C ABI declared in include/csm_gpu.h.

The engine library is loaded from the package tree (paracosm_b200/_lib); a
missing library is an error, never a silent CPU path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libcsmgpu.so"

CSM_OK = 0
CSM_EINVAL = -1
CSM_ENOMEM = -2
CSM_ECUDA = -3
CSM_ESTATE = -4
CSM_EUNSUPPORTED = -5
CSM_ETIMEOUT = -6
CSM_EDEVICE = -7

ST_OK, ST_CAPPED, ST_TIMED_OUT, ST_INVALID = 0, 1, 2, 3

ALGO_GRAPHFLOW, ALGO_TURBOFLUX, ALGO_SYMBI, ALGO_CALIG, ALGO_NEWSP = 0, 1, 2, 3, 4
MODE_BATCHED, MODE_PLAIN = 0, 1

# The reference's -a names (ParaCOSM/CSM/matching/main.cpp:740-757) and the engine algorithm behind each.
ALGORITHMS = {
    "graphflow": ALGO_GRAPHFLOW,
    "parallel_graphflow": ALGO_GRAPHFLOW,
    "turboflux": ALGO_TURBOFLUX,
    "parallel_turboflux": ALGO_TURBOFLUX,
    "symbi": ALGO_SYMBI,
    "parallel_symbi": ALGO_SYMBI,
    # CaLiG is its own program in the reference (ParaCOSM/CSM/matching/Parallel_CaLiG)
    "calig": ALGO_CALIG,
    "parallel_calig": ALGO_CALIG,
    # NewSP has its own driver in the reference (ParaCOSM/CSM/matching/Parallel_NewSP/matching/main.cpp)
    "newsp": ALGO_NEWSP,
    "parallel_newsp": ALGO_NEWSP,
}

UPDATE_DTYPE = np.dtype(
    [("type", "u1"), ("is_add", "u1"), ("pad", "<u2"), ("id1", "<u4"), ("id2", "<u4"), ("label", "<u4")]
)
RESULT_DTYPE = np.dtype(
    [("pos", "<u8"), ("neg", "<u8"), ("hash", "<u8"), ("work_bytes", "<u8"), ("latency_ns", "<u8"),
     ("status", "<u4"), ("safe", "<u4")]
)
assert UPDATE_DTYPE.itemsize == 16 and RESULT_DTYPE.itemsize == 48


class CsmCfg(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int32),
        ("homomorphism", C.c_int32),
        ("max_results", C.c_uint64),
        ("deadline_ns", C.c_uint64),
        ("hbm_budget_bytes", C.c_uint64),
        ("mode", C.c_int32),
        ("max_batch", C.c_uint32),
        ("want_hash", C.c_int32),
        ("device", C.c_int32),
        ("turboflux_compat", C.c_int32),
        ("warps_per_block", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("vertex_headroom", C.c_uint32),
        ("graphs", C.c_int32),
        ("shard_rank", C.c_uint32),
        ("shard_count", C.c_uint32),
        ("donate_every", C.c_uint32),
        ("split_deep", C.c_uint32),
        ("enum_capacity", C.c_uint32),
        ("tail_enumerate", C.c_uint32),
    ]


class CsmStats(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_uint64), ("num_edges", C.c_uint64),
        ("updates_done", C.c_uint64), ("vertex_updates", C.c_uint64), ("edge_updates", C.c_uint64),
        ("positive", C.c_uint64), ("negative", C.c_uint64), ("unsafe_updates", C.c_uint64),
        ("batches", C.c_uint64), ("kernel_launches", C.c_uint64),
        ("search_tasks", C.c_uint64), ("donated_tasks", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("pool_entries", C.c_uint64), ("pool_capacity", C.c_uint64),
        ("last_batch_ms", C.c_double), ("total_device_ms", C.c_double),
        ("index_entries", C.c_uint64), ("index_vertices", C.c_uint64),
        ("search_launches", C.c_uint64), ("search_ms", C.c_double), ("work_bytes", C.c_uint64),
        ("search_busy_ns", C.c_uint64), ("search_idle_ns", C.c_uint64), ("search_iters", C.c_uint64),
        ("search_donations", C.c_uint64), ("search_starved", C.c_uint64),
    ]


class CsmIndexInfo(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int32), ("n_qv", C.c_uint32), ("root", C.c_uint32), ("reserved", C.c_uint32),
        ("words", C.c_uint64), ("order", C.c_uint32 * 32), ("parents", C.c_uint32 * 32),
        ("d1_count", C.c_uint64), ("d2_count", C.c_uint64),
    ]


# Every symbol include/csm_gpu.h declares: (name, restype, argtypes).
_SIGNATURES = [
    ("csm_gpu_default_cfg", None, [C.POINTER(CsmCfg)]),
    ("csm_gpu_create", C.c_int, [C.POINTER(CsmCfg), C.POINTER(C.c_void_p)]),
    ("csm_gpu_set_query", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("csm_gpu_load_graph", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p]),
    ("csm_gpu_reserve_labels", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p]),
    ("csm_gpu_attach_query", C.c_int, [C.c_void_p, C.POINTER(CsmCfg), C.c_uint32, C.c_void_p, C.c_uint32,
                                       C.c_void_p, C.POINTER(C.c_void_p)]),
    ("csm_gpu_build_index", C.c_int, [C.c_void_p]),
    ("csm_gpu_initial_match", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("csm_gpu_autotune", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_float)]),
    ("csm_gpu_classify", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    ("csm_gpu_submit", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    ("csm_gpu_submit_device", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    ("csm_gpu_poll", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("csm_gpu_wait", C.c_int, [C.c_void_p, C.c_uint64]),
    ("csm_gpu_results", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p]),
    ("csm_gpu_results_device", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]),
    ("csm_gpu_stats", C.c_int, [C.c_void_p, C.POINTER(CsmStats)]),
    ("csm_gpu_probe_noalloc", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("csm_gpu_index_info", C.c_int, [C.c_void_p, C.POINTER(CsmIndexInfo)]),
    ("csm_gpu_index_flags", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64]),
    ("csm_gpu_matches", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_uint64)]),
    ("csm_gpu_stream", C.c_void_p, [C.c_void_p]),
    ("csm_gpu_search_counters", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32]),
    ("csm_gpu_kernel_launches", C.c_uint64, [C.c_void_p]),
    ("csm_gpu_destroy", None, [C.c_void_p]),
    ("csm_gpu_last_error", C.c_char_p, []),
    ("csm_gpu_strerror", C.c_char_p, [C.c_int]),
]

EXPORTED = [s[0] for s in _SIGNATURES]

_lib = None


def load_library(path: Path | str | None = None) -> C.CDLL:
    """Loads libcsmgpu.so (built by paracosm_b200.build) and types its entry points."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"CUDA engine library missing: {p} (run `python -m paracosm_b200.build`)")
    lib = C.CDLL(str(p))
    for name, res, args in _SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


class CsmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"csm error {code}: {msg}")
        self.code = code


def check(lib: C.CDLL, rc: int) -> None:
    if rc != CSM_OK:
        raise CsmError(rc, (lib.csm_gpu_last_error() or b"").decode())
