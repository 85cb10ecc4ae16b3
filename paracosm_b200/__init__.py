"""B200-native continuous subgraph matching behind ParaCOSM's plugin interface.

The CUDA engine (paracosm_b200/csrc, C ABI in include/csm_gpu.h) holds the
data graph as a label-partitioned dynamic CSR in HBM and counts, for every
edge insertion or deletion, the embeddings of a labelled query graph that
contain the updated edge, with the sequential update order's semantics.
"""
from ._abi import (ALGORITHMS, RESULT_DTYPE, ST_CAPPED, ST_INVALID, ST_OK, ST_TIMED_OUT, UPDATE_DTYPE, CsmError,
                   load_library)
from .engine import (PLUGINS, Engine, Graph, Graphflow, Parallel_Graphflow, Parallel_TurboFlux, Parrllel_SymBi, SymBi,
                     TurboFlux, matching)

__all__ = [
    "ALGORITHMS", "RESULT_DTYPE", "UPDATE_DTYPE", "ST_OK", "ST_CAPPED", "ST_TIMED_OUT", "ST_INVALID", "CsmError",
    "load_library", "Engine", "Graph", "matching", "Graphflow", "TurboFlux", "SymBi", "Parallel_Graphflow",
    "Parallel_TurboFlux", "Parrllel_SymBi", "PLUGINS",
]
