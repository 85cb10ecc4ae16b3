"""Regenerates the golden fixtures under tests/golden/ from the reference itself.

Each case is a small seeded workload (written by paracosm_b200/_bin/csm_gen)
run through the reference plugins compiled from their sources
(oracle/_ref/ref_driver, built by `make -C oracle/ref_build`) with the
sequential per-update semantics of the reference's SingleThreadUpdate loop.
The fixture keeps the inputs in the reference's text formats and, per
update, the positive / negative counts of each plugin and the match-set hash
of sequential SymBi (parsed from its --print-enum output).  index_symbi.txt
and index_turboflux.txt hold those plugins' own candidate index (root,
serialized DAG, parents, d1 / d2 flags as little-endian hex bitsets) after
preprocessing, after half of the stream and after all of it, read out of the
plugin objects by ref_driver --dump-index.  initial.json holds the
InitialMatching count the reference's own csm driver prints for the graph
before the stream.

    python tests/golden/make_golden.py          # needs the reference sources to build the driver
    python tests/golden/make_golden.py --index  # only the index fixtures
    python tests/golden/make_golden.py --initial  # only initial.json (InitialMatching counts of csm)
    python tests/golden/make_golden.py --calig    # only the calig_* cases
    python tests/golden/make_golden.py --c3shape  # only the c3_shape case
    python tests/golden/make_golden.py --selfloop # only the selfloop case

The selfloop case is a data graph with self loops (the generator never
writes them; the reference's Graph::AddEdge stores a loop's vertex twice in
its own neighbour list, ParaCOSM/CSM/graph/graph.cpp:58-76) and a query with
an edge between two vertices of one label, so that under --homo an embedding
can map that edge onto a loop.  selfloop.csv holds sequential SymBi's
per-update counts with and without --homo, on the graph with its loops and
on the same graph without them.

The c3_shape case has the shape of the 2^22-vertex SymBi benchmark at a size
the CPU finishes: 2^16 vertices, average degree 28, 16 vertex labels
Zipf(1.2), 4 edge labels, a 16-vertex dense query (average degree >= 4), an
80/20 insert/delete stream of 70,000 updates.  Its inputs are not stored: the
seeded generator rebuilds them, and params.json holds the SHA-256 of the
files it writes so that a changed generator is caught.  expected.csv lists
only the updates where some count is nonzero (every other update counts 0):
sequential SymBi's pos / neg / match-set hash with max_results 1e6, and its
pos / neg with max_results 20,000 (it stops at exactly the cap).

The calig_* cases are in the reference CaLiG program's own formats (data,
query, stream; no edge labels, insertions only, since the reference cannot
process deletion records) and hold, per update, the count of the
reference's CaLiG (oracle/_ref/calig_ref, its update loop run serially) in
expected.txt, and the lighting after its static filtering in lit.txt (one
`u v` pair per lit candidate).

Only this script reads the reference; the fixtures it writes are plain files.
"""
from __future__ import annotations

import json
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle  # noqa: E402
from paracosm_b200 import workload  # noqa: E402

GEN = ROOT / "paracosm_b200" / "_bin" / "csm_gen"

# name: (generator args, max_results, homo)
CASES = {
    "c1_small": (["--preset", "c1", "--log2-n", "11", "--updates", "300", "--seed", "11"], None, False),
    "mixed_2el": (["--preset", "c2", "--log2-n", "11", "--avg-degree", "6", "--vlabels", "3", "--zipf", "1.0",
                   "--elabels", "2", "--updates", "400", "--insert-frac", "0.7", "--seed", "12",
                   "--query", "6:sparse:1"], None, False),
    "dense_del": (["--preset", "c2", "--log2-n", "10", "--avg-degree", "10", "--vlabels", "3", "--zipf", "0",
                   "--elabels", "2", "--updates", "300", "--insert-frac", "0.6", "--seed", "13",
                   "--query", "4:dense"], None, False),
    "capped": (["--preset", "c2", "--log2-n", "11", "--avg-degree", "8", "--vlabels", "2", "--zipf", "0",
                "--elabels", "1", "--updates", "200", "--insert-frac", "0.8", "--seed", "14",
                "--query", "5:sparse:1"], 40, False),
    "homo": (["--preset", "c2", "--log2-n", "10", "--avg-degree", "8", "--vlabels", "2", "--zipf", "0",
              "--elabels", "1", "--updates", "200", "--insert-frac", "0.7", "--seed", "15",
              "--query", "4:sparse:1"], None, True),
    "zipf_8q": (["--preset", "c2", "--log2-n", "12", "--avg-degree", "8", "--vlabels", "6", "--zipf", "1.2",
                 "--elabels", "2", "--updates", "300", "--insert-frac", "0.85", "--seed", "16",
                 "--query", "8:dense"], None, False),
}

PLUGINS = [("graphflow", 1), ("symbi", 1), ("turboflux", 1), ("parallel_graphflow", 4), ("parallel_turboflux", 4),
           ("parallel_symbi", 32)]


def write_index(d: Path) -> None:
    """Writes index_<algo>.txt for one case from the reference's own index state."""
    import numpy as np

    vl, _ = workload.read_graph(d / "data.graph")
    n_up = len(workload.read_stream(d / "stream.txt"))
    ats = [0, n_up // 2, n_up]
    for algo in ("symbi", "turboflux"):
        ref = pyoracle.ref_index(d / "query.graph", d / "data.graph", d / "stream.txt", algo, ats, len(vl))
        with open(d / f"index_{algo}.txt", "w") as f:
            for at in ats:
                r = ref[at]
                f.write(f"at {at}\nroot {r['root']}\norder {' '.join(map(str, r['order']))}\n")
                for q, ps in enumerate(r["parents"]):
                    f.write(f"parents {q} {' '.join(map(str, ps))}".rstrip() + "\n")
                for k in ("d1", "d2"):
                    for q in range(len(r["order"])):
                        f.write(f"{k} {q} {np.packbits(r[k][q], bitorder='little').tobytes().hex()}\n")


REF_CSM = ROOT / "oracle" / "_ref" / "csm"
REF_CALIG = ROOT / "oracle" / "_ref" / "calig_ref"

# name: generator args (one edge label, insertions only)
CALIG_CASES = {
    # several insertions at vertices that had no neighbour in the initial graph
    "calig_sparse": ["--preset", "c2", "--log2-n", "10", "--avg-degree", "6", "--vlabels", "3", "--zipf", "0",
                     "--elabels", "1", "--updates", "300", "--insert-frac", "1.0", "--seed", "1",
                     "--query", "5:sparse:1"],
    "calig_dense": ["--preset", "c2", "--log2-n", "11", "--avg-degree", "10", "--vlabels", "2", "--zipf", "0",
                    "--elabels", "1", "--updates", "300", "--insert-frac", "1.0", "--seed", "7",
                    "--query", "6:dense"],
    "calig_tree": ["--preset", "c2", "--log2-n", "10", "--avg-degree", "8", "--vlabels", "4", "--zipf", "0",
                   "--elabels", "1", "--updates", "400", "--insert-frac", "1.0", "--seed", "27",
                   "--query", "6:sparse:2"],
    # from update 97 on the reference counts fewer matches than exist: a vertex
    # without neighbours in the initial graph keeps partial candidate maps,
    # which its later insertions do not fill (kept as a record of that defect)
    "calig_undercount": ["--preset", "c2", "--log2-n", "10", "--avg-degree", "4", "--vlabels", "2", "--zipf", "0",
                         "--elabels", "1", "--updates", "400", "--insert-frac", "1.0", "--seed", "40",
                         "--query", "5:sparse:1"],
}


def write_calig(name: str, args: list[str]) -> None:
    d = HERE / name
    tmp = HERE / f"_tmp_{name}"
    if tmp.exists():
        shutil.rmtree(tmp)
    subprocess.run([str(GEN)] + args + ["--out", str(tmp), "--calig", "--no-binary"], check=True, capture_output=True)
    d.mkdir(exist_ok=True)
    shutil.copy(tmp / "data.calig", d / "data")
    shutil.copy(tmp / "stream.calig", d / "stream")
    shutil.copy(tmp / "query_0.calig", d / "query")
    shutil.rmtree(tmp)
    r = subprocess.run([str(REF_CALIG), "-d", "data", "-q", "query", "-s", "stream", "--out", "expected.txt",
                        "--dump-li", "lit.txt"], cwd=d, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{name}: calig_ref failed: {r.stderr[-400:]}")
    (d / "params.json").write_text(json.dumps({"generator": args, "reference": "ParaCOSM/CSM/matching/"
                                               "Parallel_CaLiG/parallel_calig.cpp, serial"}, indent=1) + "\n")
    print(name, r.stderr.strip().splitlines()[-1])


def write_initial(d: Path, homo: bool) -> None:
    """initial.json: the InitialMatching count the reference's own csm driver reports per plugin."""
    out = {}
    for algo in ("graphflow", "turboflux", "symbi"):
        cmd = [str(REF_CSM), "-q", "query.graph", "-d", "data.graph", "-u", "stream.txt", "-a", algo,
               "--print-prep", "0", "--homo", "1" if homo else "0"]
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=600)
        lines = r.stdout.splitlines()
        k = lines.index("----------- Initial Matching ----------")
        out[algo] = int(lines[k + 2].split()[0])
    (d / "initial.json").write_text(json.dumps(out) + "\n")


C3_SHAPE = ["--preset", "c3", "--log2-n", "16", "--updates", "70000", "--seed", "35"]
C3_SHAPE_CAPS = (1_000_000, 20_000)


def c3_shape_files(out: Path) -> dict:
    """Generates the c3_shape inputs into `out`; returns the SHA-256 of each file."""
    import hashlib

    subprocess.run([str(GEN)] + C3_SHAPE + ["--out", str(out)], check=True, capture_output=True)
    return {f: hashlib.sha256((out / f).read_bytes()).hexdigest()
            for f in ("data.bin", "stream.bin", "query_0.graph")}


def write_c3_shape() -> None:
    d = HERE / "c3_shape"
    tmp = HERE / "_tmp_c3_shape"
    if tmp.exists():
        shutil.rmtree(tmp)
    sha = c3_shape_files(tmp)
    full, _ = pyoracle.ref_run(tmp / "query_0.graph", tmp / "data.bin", tmp / "stream.bin", "symbi",
                               max_results=C3_SHAPE_CAPS[0], want_hash=True, binary=True, timeout=3600)
    capped, _ = pyoracle.ref_run(tmp / "query_0.graph", tmp / "data.bin", tmp / "stream.bin", "symbi",
                                 max_results=C3_SHAPE_CAPS[1], binary=True, timeout=3600)
    shutil.rmtree(tmp)
    d.mkdir(exist_ok=True)
    n = len(full)
    with open(d / "expected.csv", "w") as f:
        f.write("idx,symbi_pos,symbi_neg,symbi_hash,symbi_cap_pos,symbi_cap_neg\n")
        for i in range(n):
            a, c = full[i], capped[i]
            if a["pos"] or a["neg"] or c["pos"] or c["neg"]:
                f.write(f"{i},{a['pos']},{a['neg']},{a['hash']},{c['pos']},{c['neg']}\n")
    (d / "params.json").write_text(json.dumps({
        "generator": C3_SHAPE, "updates": n, "max_results": C3_SHAPE_CAPS[0], "max_results_capped": C3_SHAPE_CAPS[1],
        "sha256": sha, "reference": "ParaCOSM/CSM/matching/SymBi (sequential), SingleThreadUpdate order"},
        indent=1) + "\n")
    print("c3_shape updates", n, "nonzero", sum(1 for i in range(n) if full[i]["pos"] or full[i]["neg"]))


SELFLOOP = ["--preset", "c2", "--log2-n", "10", "--avg-degree", "8", "--vlabels", "2", "--zipf", "0",
            "--elabels", "1", "--updates", "300", "--insert-frac", "0.8", "--seed", "17", "--query", "4:dense"]


def write_selfloop() -> None:
    import random

    d = HERE / "selfloop"
    tmp = HERE / "_tmp_selfloop"
    if tmp.exists():
        shutil.rmtree(tmp)
    subprocess.run([str(GEN)] + SELFLOOP + ["--out", str(tmp), "--text"], check=True, capture_output=True)
    d.mkdir(exist_ok=True)
    lines = (tmp / "data.graph").read_text().splitlines()
    n = sum(1 for x in lines if x.startswith("v "))
    rng = random.Random(17)
    loops = [f"e {v} {v} 0" for v in sorted(rng.sample(range(n), 80))]
    (d / "data.graph").write_text("\n".join(lines + loops) + "\n")
    (d / "data_noloop.graph").write_text("\n".join(lines) + "\n")
    shutil.copy(tmp / "stream.txt", d / "stream.txt")
    shutil.copy(tmp / "query_0.graph", d / "query.graph")
    shutil.rmtree(tmp)
    cols = {}
    for name, data, homo in (("loop", "data.graph", False), ("loop_homo", "data.graph", True),
                             ("noloop_homo", "data_noloop.graph", True)):
        rows, _ = pyoracle.ref_run(d / "query.graph", d / data, d / "stream.txt", "symbi", homo=homo, timeout=600)
        cols[name] = rows
    with open(d / "selfloop.csv", "w") as f:
        f.write("idx,pos,neg,homo_pos,homo_neg,homo_noloop_pos,homo_noloop_neg\n")
        for i in range(len(cols["loop"])):
            a, b, c = cols["loop"][i], cols["loop_homo"][i], cols["noloop_homo"][i]
            f.write(f"{i},{a['pos']},{a['neg']},{b['pos']},{b['neg']},{c['pos']},{c['neg']}\n")
    (d / "params.json").write_text(json.dumps({"generator": SELFLOOP, "self_loops": 80, "label": 0,
                                               "reference": "ParaCOSM/CSM/matching/SymBi (sequential)"}, indent=1) + "\n")
    diff = sum(1 for i in range(len(cols["loop"])) if cols["loop_homo"][i]["pos"] != cols["noloop_homo"][i]["pos"]
               or cols["loop_homo"][i]["neg"] != cols["noloop_homo"][i]["neg"])
    print("selfloop updates", len(cols["loop"]), "homo counts changed by the loops at", diff, "updates")


def main() -> None:
    if "--selfloop" in sys.argv:
        write_selfloop()
        return
    if "--c3shape" in sys.argv:
        write_c3_shape()
        return
    if "--calig" in sys.argv:
        for name, args in CALIG_CASES.items():
            write_calig(name, args)
        return
    if "--initial" in sys.argv:
        for name, (_, _, homo) in CASES.items():
            write_initial(HERE / name, homo)
            print(name, (HERE / name / "initial.json").read_text().strip())
        return
    if "--index" in sys.argv:
        for name in CASES:
            write_index(HERE / name)
            print(name, "index fixtures")
        return
    for name, (args, cap, homo) in CASES.items():
        d = HERE / name
        tmp = HERE / f"_tmp_{name}"
        if tmp.exists():
            shutil.rmtree(tmp)
        subprocess.run([str(GEN)] + args + ["--out", str(tmp), "--text"], check=True, capture_output=True)
        d.mkdir(exist_ok=True)
        shutil.copy(tmp / "data.graph", d / "data.graph")
        shutil.copy(tmp / "stream.txt", d / "stream.txt")
        shutil.copy(tmp / "query_0.graph", d / "query.graph")
        shutil.rmtree(tmp)
        cols = {}
        for algo, threads in PLUGINS:
            want_hash = algo in ("symbi", "turboflux")
            kw = {"threads": threads, "want_hash": want_hash}
            if cap is not None:
                kw["max_results"] = cap
            try:
                rows, _ = pyoracle.ref_run(d / "query.graph", d / "data.graph", d / "stream.txt", algo, timeout=600,
                                           homo=homo, **kw)
            except Exception as exc:  # a reference defect (e.g. exit on a deletion) is recorded, not fatal
                print(f"{name}/{algo}: {exc}".splitlines()[0])
                continue
            cols[algo] = rows
        n = len(workload.read_stream(d / "stream.txt"))
        with open(d / "expected.csv", "w") as f:
            hdr = ["idx"]
            for algo, _ in PLUGINS:
                if algo in cols:
                    hdr += [f"{algo}_pos", f"{algo}_neg"]
                    if algo in ("symbi", "turboflux"):
                        hdr += [f"{algo}_hash"]
            f.write(",".join(hdr) + "\n")
            for i in range(n):
                row = [str(i)]
                for algo, _ in PLUGINS:
                    if algo in cols:
                        r = cols[algo][i] if i < len(cols[algo]) else None
                        row += [str(r["pos"]) if r is not None else "", str(r["neg"]) if r is not None else ""]
                        if algo in ("symbi", "turboflux"):
                            row += [str(r["hash"]) if r is not None else ""]
                f.write(",".join(row) + "\n")
        (d / "params.json").write_text(json.dumps({"max_results": cap, "homo": homo, "generator": args,
                                                   "plugins": [a for a, _ in PLUGINS if a in cols]}, indent=1))
        write_index(d)
        write_initial(d, homo)
        print(name, "updates", n, "plugins", list(cols))


if __name__ == "__main__":
    main()
