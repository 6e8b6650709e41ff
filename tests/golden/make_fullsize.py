"""Generates tests/golden/fullsize.json: the compiled reference's per-coloring
raw counts on the benchmark workloads at their full sizes.

For each workload (R-MAT graph from subgraph_b200.synth -- numpy only, the
same generator the benchmark uses -- and the workload's tree template) it
runs oracle/_ref/ref_oracle (the reference's own CountMat::colorCounting,
built from its sources by oracle/build_ref.sh) for two colorings seeded
srand(7) and srand(8) with all host cores on the counting loops, and stores
the graph's size and digest (so a test can check that it regenerated the
same graph), the two full-precision raw counts and the estimate
CountMat::compute would print for them (no automorphism division, as in the
reference CLI).

Usage: python tests/golden/make_fullsize.py   (needs oracle/_ref/ref_oracle)
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from subgraph_b200 import synth  # noqa: E402

TEMPLATES = {
    "p3": (3, [(0, 1), (1, 2)]),
    "tree5": (5, [(0, 1), (1, 2), (2, 3), (1, 4)]),
    "spider7": (7, [(0, 1), (1, 2), (0, 3), (3, 4), (0, 5), (5, 6)]),
    "tree12": (12, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 6), (6, 7), (2, 8), (4, 9), (5, 10), (10, 11)]),
}
WORKLOADS = [
    ("p3_rmat16_ef16", 16, 16, "p3"),
    ("tree5_rmat20_ef6", 20, 6, "tree5"),
    ("spider7_rmat21_ef8", 21, 8, "spider7"),
    ("tree12_rmat20_ef8", 20, 8, "tree12"),
]
SEED, NCOL = 7, 2


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/ref_oracle is missing: run oracle/build_ref.sh first")
    threads = os.cpu_count() or 1
    out = {"seed": SEED, "ncol": NCOL, "graph_seed": 1, "initiator": [0.57, 0.19, 0.19], "workloads": {}}
    with tempfile.TemporaryDirectory() as tmp:
        for name, scale, ef, tname in WORKLOADS:
            V, src, dst = synth.rmat_edges(scale, ef, seed=1)
            gpath = os.path.join(tmp, f"{name}.txt")
            synth.write_edge_list(gpath, V, src, dst)
            n, edges = TEMPLATES[tname]
            tpath = os.path.join(tmp, f"{tname}.t")
            with open(tpath, "w") as f:
                f.write(f"{n}\n{len(edges)}\n" + "".join(f"{a} {b}\n" for a, b in edges))
            R = O.run_ref(gpath, tpath, NCOL, SEED, os.path.join(tmp, "o_" + name), threads=threads, light=True)
            raw = [float(x) for x in R["raw"]]
            out["workloads"][name] = {
                "scale": scale, "edge_factor": ef, "template": tname, "n": n, "edges": [list(e) for e in edges],
                "V": V, "E": int(len(src)), "digest": synth.edges_digest(V, src, dst), "raw": raw,
                "estimate": O.estimate(R["raw"], n, 1),
                "ref_seconds_per_coloring": float(R["times"].mean()), "ref_threads": threads,
            }
            print(name, raw, f"{R['times'].mean():.2f} s/coloring", flush=True)
    with open(os.path.join(HERE, "fullsize.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
