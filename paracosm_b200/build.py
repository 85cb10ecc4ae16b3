"""Builds the native parts in-tree.

    python -m paracosm_b200.build            # engine + host tools + oracle (+ reference if present)

Outputs (git-ignored, but they travel with the working tree):
    paracosm_b200/_lib/libcsmgpu.so   CUDA engine behind include/csm_gpu.h (sm_100a)
    paracosm_b200/_bin/csm            csm driver (reference command line) over the engine
    paracosm_b200/_bin/csm_serve      serving loop (standing queries, streamed updates, continuous batching)
    paracosm_b200/_bin/csm_gen        seeded workload generator
    paracosm_b200/_bin/calig          the reference's CaLiG program (its formats and output) over the engine
    oracle/_build/                    CPU restatement used as the checker
    oracle/_ref/                      the reference compiled from its sources (checker / CPU baseline)
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
LIB = PKG / "_lib"
BIN = PKG / "_bin"
OBJ = PKG / "_lib" / "obj"


def reference_sources() -> Path | None:
    """ParaCOSM/CSM of the reference checkout, when it is present: $PARACOSM_REFERENCE
    (the checkout root), else BASELINE.json's reference_path.  The reference is
    only compiled as the checker and CPU baseline (oracle/_ref)."""
    import json

    root = os.environ.get("PARACOSM_REFERENCE")
    if not root:
        try:
            root = json.loads((ROOT / "BASELINE.json").read_text()).get("reference_path")
        except (OSError, ValueError):
            root = None
    if not root:
        return None
    src = Path(root) / "ParaCOSM" / "CSM"
    return src if src.exists() else None

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", CXX] + ARCH

CU_SOURCES = ["csm_api.cu", "csm_kernels.cu", "csm_search.cu", "csm_index.cu", "csm_noalloc.cu"]
HEADERS = [CSRC / h for h in ("csm_internal.cuh", "csm_kernels.cuh", "csm_index.cuh", "csm_host.cuh")] + [
    ROOT / "include" / "csm_gpu.h"
]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], cwd: Path | None = None) -> None:
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_engine(force: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    objs = []
    jobs = []
    for src in CU_SOURCES:
        o = OBJ / (Path(src).stem + ".o")
        objs.append(o)
        if force or _stale(o, [CSRC / src] + HEADERS):
            jobs.append([NVCC] + NVFLAGS + ["-c", str(CSRC / src), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=len(CU_SOURCES)) as ex:
        list(ex.map(_run, jobs))
    lib = LIB / "libcsmgpu.so"
    if force or _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-ccbin", CXX, "-o", str(lib)] + [str(o) for o in objs] + ["-lcudart"])
    return lib


def build_host(force: bool = False) -> None:
    BIN.mkdir(parents=True, exist_ok=True)
    common = [HOST / "graph_io.cpp"]
    gen = BIN / "csm_gen"
    gen_src = [HOST / "csm_gen.cpp", HOST / "workload.cpp", HOST / "calig_io.cpp"] + common
    if force or _stale(gen, gen_src + [HOST / "workload.h", HOST / "graph_io.h", HOST / "calig_io.h"]):
        _run([CXX, "-std=c++17", "-O3", "-fopenmp", "-o", str(gen)] + [str(s) for s in gen_src])
    link = ["-L", str(LIB), "-lcsmgpu", f"-Wl,-rpath,{LIB}", "-Wl,-rpath,$ORIGIN/../_lib"]
    srv = BIN / "csm_serve"
    srv_src = [HOST / "csm_serve.cpp", HOST / "serve.cpp"] + common
    deps = srv_src + [HOST / "serve.h", HOST / "graph_io.h", ROOT / "include" / "csm_gpu.h", LIB / "libcsmgpu.so"]
    if force or _stale(srv, deps):
        _run([CXX, "-std=c++17", "-O3", "-pthread", "-I", str(ROOT / "include"), "-o", str(srv)]
             + [str(s) for s in srv_src] + link)
    drv = BIN / "csm"
    drv_src = [HOST / "csm_main.cpp", HOST / "plugins.cpp"] + common
    if (HOST / "csm_main.cpp").exists():
        deps = drv_src + [HOST / "plugins.h", HOST / "graph_io.h", ROOT / "include" / "csm_gpu.h", LIB / "libcsmgpu.so"]
        if force or _stale(drv, deps):
            _run([CXX, "-std=c++17", "-O3", "-I", str(ROOT / "include"), "-o", str(drv)] + [str(s) for s in drv_src]
                 + ["-L", str(LIB), "-lcsmgpu", f"-Wl,-rpath,{LIB}", "-Wl,-rpath,$ORIGIN/../_lib"])
    cal = BIN / "calig"
    cal_src = [HOST / "calig_main.cpp", HOST / "calig_io.cpp", HOST / "plugins.cpp"] + common
    deps = cal_src + [HOST / "calig_io.h", HOST / "plugins.h", HOST / "graph_io.h", ROOT / "include" / "csm_gpu.h",
                      LIB / "libcsmgpu.so"]
    if force or _stale(cal, deps):
        _run([CXX, "-std=c++17", "-O3", "-I", str(ROOT / "include"), "-o", str(cal)] + [str(s) for s in cal_src] + link)


def build_oracle(force: bool = False) -> None:
    env = dict(os.environ, CXX=CXX)
    _run(["make", "-C", str(ROOT / "oracle")] + (["-B"] if force else []), cwd=ROOT)
    ref = reference_sources()
    if ref is not None:
        _run(["make", "-C", str(ROOT / "oracle" / "ref_build"), f"REF={ref}", "-j8"], cwd=ROOT)
    del env


def build_all(force: bool = False) -> None:
    build_engine(force)
    build_host(force)
    build_oracle(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", LIB / "libcsmgpu.so")
