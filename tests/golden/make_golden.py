"""Generates tests/golden/golden.npz from the compiled reference.

Runs oracle/_ref/ref_oracle (the reference's own CountMat / CSCGraph /
EdgeList / DivideTemplates / IndexSys objects, built by oracle/build_ref.sh)
on small seeded graphs and templates and stores what it produced:
  - the edge list given to it (text form is re-created by the tests),
  - its CSC arrays,
  - its sub-template list and IndexSys tables (as arrays or SHA-256 digests),
  - the colors of every coloring (srand(seed + c), one thread),
  - the full-precision raw count of every coloring,
  - SHA-256 digests of every sub-template table of coloring 0 (column-major
    float32 bytes, exactly as DataTableColMajor holds them).

Usage: python tests/golden/make_golden.py   (needs oracle/_ref/ref_oracle)
"""
from __future__ import annotations

import hashlib
import json
import os
import random
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

TEMPLATES = {
    "p3": (3, [(0, 1), (1, 2)]),
    "tree5": (5, [(0, 1), (1, 2), (2, 3), (1, 4)]),
    "spider7": (7, [(0, 1), (1, 2), (0, 3), (3, 4), (0, 5), (5, 6)]),
    "tree12": (12, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 6), (6, 7), (2, 8), (4, 9), (5, 10), (10, 11)]),
    "p2": (2, [(0, 1)]),
    "star4": (4, [(0, 1), (0, 2), (0, 3)]),
    "p3_mid": (3, [(1, 0), (1, 2)]),
}


def rmat_edges(scale: int, ef: int, seed: int, a=0.57, b=0.19, c=0.19):
    """Plain R-MAT with a seeded numpy generator, symmetrised and deduplicated."""
    rng = np.random.default_rng(seed)
    n = 1 << scale
    m = ef * n
    u = np.zeros(m, np.int64)
    v = np.zeros(m, np.int64)
    for level in range(scale):
        r = rng.random(m)
        bu = (r >= a + b).astype(np.int64)
        bv = (((r >= a) & (r < a + b)) | (r >= a + b + c)).astype(np.int64)
        u |= bu << level
        v |= bv << level
    perm = rng.permutation(n)
    u, v = perm[u], perm[v]
    keep = u != v
    lo = np.minimum(u[keep], v[keep])
    hi = np.maximum(u[keep], v[keep])
    e = np.unique(lo * n + hi)
    lo, hi = (e // n).astype(np.int32), (e % n).astype(np.int32)
    if max(lo.max(), hi.max()) != n - 1:      # keep max id = V-1 (no hole removal)
        top = max(lo.max(), hi.max())
        lo = np.where(lo == top, n - 1, lo)
        hi = np.where(hi == top, n - 1, hi)
    return n, lo, hi


def prufer_tree(n: int, rng: random.Random):
    seq = [rng.randrange(n) for _ in range(n - 2)]
    deg = [1] * n
    for x in seq:
        deg[x] += 1
    edges = []
    for x in seq:
        for leaf in range(n):
            if deg[leaf] == 1:
                edges.append((leaf, x))
                deg[leaf] -= 1
                deg[x] -= 1
                break
    u = [i for i in range(n) if deg[i] == 1]
    edges.append((u[0], u[1]))
    return edges


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def write_graph(path, V, src, dst):
    with open(path, "w") as f:
        f.write(f"{V}\n{len(src)}\n")
        f.write("".join(f"{a} {b}\n" for a, b in zip(src, dst)))


def write_template(path, n, edges):
    with open(path, "w") as f:
        f.write(f"{n}\n{len(edges)}\n")
        f.write("".join(f"{a} {b}\n" for a, b in edges))


def run_case(tmp, name, V_decl, src, dst, tname, n, edges, ncol, seed, tables=True, aut=False):
    g = os.path.join(tmp, f"{name}.txt")
    t = os.path.join(tmp, f"{name}_{tname}.t")
    write_graph(g, V_decl, src, dst)
    write_template(t, n, edges)
    out = os.path.join(tmp, f"out_{name}_{tname}")
    # splitCSC(4*threads) divides by V/(4*threads) (CSCGraph.hpp:199,207): keep it >= 1
    thr = 1 if V_decl < 64 else 4
    R = O.run_ref(g, t, ncol, seed, out, threads=thr, dump_tables=tables, automorphisms=aut)
    case = {"graph": name, "template": tname, "n": n, "edges": np.array(edges, np.int32).reshape(-1, 2),
            "ncol": ncol, "seed": seed, "raw": R["raw"], "V": R["V"], "aut": R["aut"]}
    case["colors"] = R["colors"]
    subs = []
    for s in R["subs"]:
        d = {k: s[k] for k in ("size", "main", "aux", "parent", "L", "S")}
        if s["L"] * max(s["S"], 1) <= 256:
            d["c2c"] = s["c2c"].tolist()
            if s["size"] > 1:
                d["msplit"] = s["msplit"].tolist()
                d["asplit"] = s["asplit"].tolist()
        else:
            d["c2c_sha"] = sha(s["c2c"])
            if s["size"] > 1:
                d["msplit_sha"] = sha(s["msplit"].astype(np.int32))
                d["asplit_sha"] = sha(s["asplit"].astype(np.int32))
        subs.append(d)
    case["subs"] = subs
    case["table_sha"] = {int(s): sha(T) for s, T in R["tables"].items()}
    if "raw_dump" in R:
        case["raw_dump"] = R["raw_dump"]
    return case, R


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/ref_oracle is missing: run oracle/build_ref.sh first")
    rng = random.Random(2024)
    graphs = {}
    # hand-made graph: duplicate edges, a self loop, an isolated vertex, max id = V-1
    graphs["tiny"] = (12, np.array([0, 1, 1, 2, 3, 3, 4, 5, 6, 0, 2, 7, 8, 9, 9, 4, 10], np.int32),
                      np.array([1, 2, 2, 3, 4, 5, 6, 6, 7, 4, 2, 9, 9, 11, 10, 8, 11], np.int32))
    # declared V larger than used ids -> hole removal renumbers and shrinks V
    graphs["holes"] = (20, np.array([0, 2, 2, 5, 7, 9, 11, 5], np.int32),
                       np.array([2, 5, 7, 9, 11, 13, 13, 13], np.int32))
    V10, s10, d10 = rmat_edges(10, 8, seed=1)
    graphs["rmat10"] = (V10, s10, d10)
    V12, s12, d12 = rmat_edges(12, 8, seed=2)
    graphs["rmat12"] = (V12, s12, d12)

    cases = []
    with tempfile.TemporaryDirectory() as tmp:
        for tn in ("p3", "star4", "p2", "p3_mid", "tree5"):
            c, _ = run_case(tmp, "tiny", *graphs["tiny"], tn, *TEMPLATES[tn], ncol=3, seed=7, aut=True)
            cases.append(c)
        for tn in ("p3", "tree5"):
            c, _ = run_case(tmp, "holes", *graphs["holes"], tn, *TEMPLATES[tn], ncol=2, seed=11, aut=True)
            cases.append(c)
        for tn in ("p3", "tree5", "spider7", "tree12", "p2"):
            c, _ = run_case(tmp, "rmat10", *graphs["rmat10"], tn, *TEMPLATES[tn], ncol=3, seed=7,
                            aut=TEMPLATES[tn][0] <= 8)
            cases.append(c)
        c, _ = run_case(tmp, "rmat12", *graphs["rmat12"], "tree12", *TEMPLATES["tree12"], ncol=2, seed=7,
                        tables=False)
        cases.append(c)
        # random trees of 3..10 vertices (edges in Pruefer decode order), one or two colorings each
        for i in range(16):
            n = rng.randint(3, 10)
            edges = prufer_tree(n, rng)
            tn = f"rand{i}"
            c, _ = run_case(tmp, "rmat10", *graphs["rmat10"], tn, n, edges, ncol=2, seed=100 + i, tables=False,
                            aut=n <= 8)
            cases.append(c)
    arrays = {}
    meta = {"graphs": {}, "cases": []}
    for gname, (V, s, d) in graphs.items():
        arrays[f"g_{gname}_src"] = s
        arrays[f"g_{gname}_dst"] = d
        meta["graphs"][gname] = {"V_declared": int(V), "E": int(len(s))}
    for i, c in enumerate(cases):
        key = f"c{i}"
        arrays[f"{key}_raw"] = np.asarray(c["raw"], np.float64)
        arrays[f"{key}_colors"] = np.asarray(c["colors"], np.int8)
        arrays[f"{key}_edges"] = c["edges"]
        m = {k: c[k] for k in ("graph", "template", "n", "ncol", "seed", "V", "aut", "subs", "table_sha")}
        m["key"] = key
        if "raw_dump" in c:
            m["raw_dump"] = c["raw_dump"]
        meta["cases"].append(m)
    # reference CSC arrays of each graph (from its first case's dump)
    with tempfile.TemporaryDirectory() as tmp:
        for gname, (V, s, d) in graphs.items():
            g = os.path.join(tmp, "g.txt")
            t = os.path.join(tmp, "t.t")
            write_graph(g, V, s, d)
            write_template(t, *TEMPLATES["p3"])
            R = O.run_ref(g, t, 1, 1, os.path.join(tmp, "o_" + gname), threads=1 if V < 64 else 4)
            arrays[f"g_{gname}_csc_col"] = R["col"]
            arrays[f"g_{gname}_csc_row"] = R["row"]
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, sort_keys=True, separators=(",", ":"))
    print(f"wrote {len(cases)} cases")


if __name__ == "__main__":
    main()
