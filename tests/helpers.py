"""Shared test helpers: golden fixtures, text files, templates, device checks."""
from __future__ import annotations

import json
import os
import random
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN_DIR = os.path.join(HERE, "golden")

TEMPLATES = {
    "p3": (3, [(0, 1), (1, 2)]),
    "tree5": (5, [(0, 1), (1, 2), (2, 3), (1, 4)]),
    "spider7": (7, [(0, 1), (1, 2), (0, 3), (3, 4), (0, 5), (5, 6)]),
    "tree12": (12, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 6), (6, 7), (2, 8), (4, 9), (5, 10), (10, 11)]),
    "p2": (2, [(0, 1)]),
    "star4": (4, [(0, 1), (0, 2), (0, 3)]),
    "p3_mid": (3, [(1, 0), (1, 2)]),
}


@dataclass
class Case:
    key: str
    graph: str
    template: str
    n: int
    edges: list
    ncol: int
    seed: int
    V: int
    aut: int
    raw: np.ndarray
    colors: np.ndarray
    subs: list
    table_sha: dict
    raw_dump: float | None


class Golden:
    def __init__(self):
        self.meta = json.load(open(os.path.join(GOLDEN_DIR, "golden.json")))
        self.arr = dict(np.load(os.path.join(GOLDEN_DIR, "golden.npz")))
        self.cases = []
        for m in self.meta["cases"]:
            k = m["key"]
            self.cases.append(Case(
                key=k, graph=m["graph"], template=m["template"], n=m["n"],
                edges=[tuple(map(int, e)) for e in self.arr[f"{k}_edges"]], ncol=m["ncol"], seed=m["seed"],
                V=m["V"], aut=m["aut"], raw=self.arr[f"{k}_raw"], colors=self.arr[f"{k}_colors"].astype(np.int32),
                subs=m["subs"], table_sha={int(a): b for a, b in m["table_sha"].items()},
                raw_dump=m.get("raw_dump")))

    def graph(self, name):
        """(V_declared, src, dst, csc_col, csc_row) of a fixture graph."""
        g = self.meta["graphs"][name]
        return (g["V_declared"], self.arr[f"g_{name}_src"], self.arr[f"g_{name}_dst"],
                self.arr[f"g_{name}_csc_col"], self.arr[f"g_{name}_csc_row"])

    def write_graph(self, name, path):
        V, s, d, _, _ = self.graph(name)
        write_graph(path, V, s, d)


def write_graph(path, V, src, dst):
    with open(path, "w") as f:
        f.write(f"{V}\n{len(src)}\n")
        f.write("".join(f"{a} {b}\n" for a, b in zip(src, dst)))


def write_template(path, n, edges):
    with open(path, "w") as f:
        f.write(f"{n}\n{len(edges)}\n")
        f.write("".join(f"{a} {b}\n" for a, b in edges))


def sha(a: np.ndarray) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


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


def rel(a, b):
    a, b = float(a), float(b)
    return abs(a - b) / max(abs(b), 1e-300)


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@dataclass
class FlagCase:
    key: str
    variant: str        # spmv | orig | csr_spmv | csr_orig
    graph: str
    template: str
    n: int
    edges: list
    ncol: int
    seed: int
    V: int
    csr: bool
    is_pruned: int
    use_spmm: int
    raw: np.ndarray
    colors: np.ndarray
    table_sha: dict


class GoldenFlags:
    """The compiled reference's results for the CountMat flag variants and the
    CSR input path (tests/golden/make_golden_flags.py)."""

    def __init__(self):
        self.meta = json.load(open(os.path.join(GOLDEN_DIR, "golden_flags.json")))
        self.arr = dict(np.load(os.path.join(GOLDEN_DIR, "golden_flags.npz")))
        self.cases = []
        for m in self.meta["cases"]:
            k = m["key"]
            self.cases.append(FlagCase(
                key=k, variant=m["variant"], graph=m["graph"], template=m["template"], n=m["n"],
                edges=[tuple(e) for e in m["edges"]], ncol=m["ncol"], seed=m["seed"], V=m["V"], csr=m["csr"],
                is_pruned=m["is_pruned"], use_spmm=m["use_spmm"], raw=self.arr[f"{k}_raw"],
                colors=self.arr[f"{k}_colors"].astype(np.int32),
                table_sha={int(a): b for a, b in m["table_sha"].items()}))

    def edges(self, name):
        g = self.meta["graphs"][name]
        return g["V_declared"], self.arr[f"g_{name}_src"], self.arr[f"g_{name}_dst"]

    def csr(self, name):
        return self.arr[f"g_{name}_csr_row"], self.arr[f"g_{name}_csr_col"]


def sha_nan(a: np.ndarray) -> str:
    """SHA-256 of a float32 table with every NaN written as one canonical NaN."""
    import hashlib
    a = np.array(a, np.float32, copy=True)
    a[np.isnan(a)] = np.float32("nan")
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def same_raw(a, b, tol=0.0) -> bool:
    """Raw counts equal within a relative tolerance; inf and NaN must match."""
    a, b = float(a), float(b)
    if np.isnan(b) or np.isinf(b):
        return (np.isnan(a) and np.isnan(b)) or a == b
    return abs(a - b) <= tol * max(abs(b), 1e-300)
