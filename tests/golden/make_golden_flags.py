"""Generates tests/golden/golden_flags.{json,npz}: the compiled reference's
results for the CountMat flag variants and the CSR input path.

Runs oracle/_ref/ref_oracle (the reference's own CountMat / CSCGraph /
CSRGraph / EdgeList / DivideTemplates / IndexSys objects, built by
oracle/build_ref.sh) with
  spmv      isPruned=1 useSPMM=0 on the CSCGraph (countNonBottomePruned,
            CountMat.cpp:325-554: one SpMV per aux column)
  orig      isPruned=0 on the CSCGraph (countNonBottomeOriginal,
            CountMat.cpp:851-977: the SpMV buffer _bufVec is never cleared,
            so it accumulates over splits, sub-templates and colorings)
  csr_spmv  isPruned=1 useSPMM=0 on a CSRGraph (SpMVNaiveFull,
            CSRGraph.cpp:190-208: neighbours in edge-file insertion order)
  csr_orig  isPruned=0 on a CSRGraph (a fresh SpMV per split)
and stores, per case, the raw count of every coloring (the colorings run one
after another on one CountMat, srand(seed + c)), SHA-256 digests of every
sub-template table of coloring 0 (column-major float32, as DataTableColMajor
holds them, NaNs canonicalised), and for the CSR graphs the reference's CSR
arrays.  The isPruned=0 CSC results grow without bound from coloring to
coloring (the accumulating buffer) and reach inf and NaN: that is the
reference's output, and the fixtures keep it.

Graphs: the hand-made graph and R-MAT scale 10 of make_golden.py, and the
same R-MAT edges in a shuffled order with random orientation (so the CSR
neighbour order differs from the CSC's ascending order).

Usage: python tests/golden/make_golden_flags.py   (needs oracle/_ref/ref_oracle)
"""
from __future__ import annotations

import hashlib
import importlib.util
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "make_golden.py"))
MG = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MG)

VARIANTS = {
    "spmv": dict(is_pruned=1, use_spmm=0, csr=False),
    "orig": dict(is_pruned=0, use_spmm=1, csr=False),
    "csr_spmv": dict(is_pruned=1, use_spmm=0, csr=True),
    "csr_orig": dict(is_pruned=0, use_spmm=1, csr=True),
}


def sha(a: np.ndarray) -> str:
    """SHA-256 of a float32 table with every NaN written as one canonical NaN
    (x86 and the GPU produce different NaN bit patterns for inf * 0)."""
    a = np.array(a, np.float32, copy=True)
    a[np.isnan(a)] = np.float32("nan")
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/ref_oracle is missing: run oracle/build_ref.sh first")
    graphs = {}
    graphs["tiny"] = (12, np.array([0, 1, 1, 2, 3, 3, 4, 5, 6, 0, 2, 7, 8, 9, 9, 4, 10], np.int32),
                      np.array([1, 2, 2, 3, 4, 5, 6, 6, 7, 4, 2, 9, 9, 11, 10, 8, 11], np.int32))
    V10, s10, d10 = MG.rmat_edges(10, 8, seed=1)
    graphs["rmat10"] = (V10, s10, d10)
    rng = np.random.default_rng(99)
    order = rng.permutation(len(s10))
    flip = rng.random(len(s10)) < 0.5
    ss, dd = s10[order].copy(), d10[order].copy()
    ss[flip], dd[flip] = d10[order][flip], s10[order][flip]
    graphs["rmat10s"] = (V10, ss.astype(np.int32), dd.astype(np.int32))

    plan = [
        ("spmv", "tiny", ("p3", "tree5"), 3, 7),
        ("spmv", "rmat10", ("tree5", "spider7", "tree12"), 2, 7),
        ("orig", "tiny", ("p3", "star4", "tree5", "p2"), 3, 7),
        ("orig", "rmat10", ("p3", "tree5", "spider7"), 3, 7),
        ("orig", "rmat10", ("tree12",), 2, 9),
        ("csr_spmv", "tiny", ("p3", "tree5"), 3, 7),
        ("csr_spmv", "rmat10s", ("tree5", "spider7", "tree12"), 2, 7),
        ("csr_orig", "tiny", ("p3", "tree5"), 3, 7),
        ("csr_orig", "rmat10s", ("tree5", "spider7"), 2, 7),
    ]
    arrays, meta = {}, {"graphs": {}, "cases": []}
    csr_seen = set()
    with tempfile.TemporaryDirectory() as tmp:
        for variant, gname, tnames, ncol, seed in plan:
            V, src, dst = graphs[gname]
            gpath = os.path.join(tmp, f"{gname}.txt")
            MG.write_graph(gpath, V, src, dst)
            for tn in tnames:
                n, edges = MG.TEMPLATES[tn]
                tpath = os.path.join(tmp, f"{tn}.t")
                MG.write_template(tpath, n, edges)
                out = os.path.join(tmp, f"out_{variant}_{gname}_{tn}")
                thr = 1 if V < 64 else 4
                R = O.run_ref(gpath, tpath, ncol, seed, out, threads=thr, dump_tables=True, **VARIANTS[variant])
                key = f"f{len(meta['cases'])}"
                arrays[f"{key}_raw"] = np.asarray(R["raw"], np.float64)
                arrays[f"{key}_colors"] = np.asarray(R["colors"], np.int8)
                meta["cases"].append({
                    "key": key, "variant": variant, "graph": gname, "template": tn, "n": n,
                    "edges": [list(e) for e in edges], "ncol": ncol, "seed": seed, "V": int(R["V"]),
                    **VARIANTS[variant],
                    "table_sha": {int(s): sha(T) for s, T in R["tables"].items()},
                })
                if VARIANTS[variant]["csr"] and gname not in csr_seen:
                    arrays[f"g_{gname}_csr_row"] = R["csr_row"]
                    arrays[f"g_{gname}_csr_col"] = R["csr_col"]
                    csr_seen.add(gname)
    for gname, (V, s, d) in graphs.items():
        arrays[f"g_{gname}_src"] = s
        arrays[f"g_{gname}_dst"] = d
        meta["graphs"][gname] = {"V_declared": int(V), "E": int(len(s))}
    np.savez_compressed(os.path.join(HERE, "golden_flags.npz"), **arrays)
    with open(os.path.join(HERE, "golden_flags.json"), "w") as f:
        json.dump(meta, f, sort_keys=True, separators=(",", ":"))
    print(f"wrote {len(meta['cases'])} cases")


if __name__ == "__main__":
    main()
