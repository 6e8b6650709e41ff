"""ctypes wrapper of the CPU oracle (oracle/sg_oracle.c) and the reference dumps.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product library never
imports this module.

The oracle restates the reference's color-coding path (see the header of
sg_oracle.c for the file:line of every piece).  ``load_ref_dump`` reads the
directory written by oracle/_ref/ref_oracle (the compiled reference).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build(force: bool = False) -> str:
    """Compile sg_oracle.c into oracle/liboracle.so (no FMA contraction)."""
    src = os.path.join(HERE, "sg_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=c99",
                               "-o", LIB_PATH, src, "-lm"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, u32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32
        L.orc_glibc_rand.argtypes = [u32, i64, vp]
        L.orc_color.argtypes = [u32, i32, i32, vp]
        L.orc_csc_build.argtypes = [i32, i32, vp, vp, vp, vp, vp]
        L.orc_csc_build.restype = ctypes.c_int
        L.orc_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int]
        L.orc_plan_create.restype = vp
        L.orc_plan_destroy.argtypes = [vp]
        L.orc_plan_nsub.argtypes = [vp]
        L.orc_plan_k.argtypes = [vp]
        L.orc_plan_aut.argtypes = [vp]
        L.orc_plan_sub.argtypes = [vp, ctypes.c_int, vp]
        L.orc_plan_tables.argtypes = [vp, ctypes.c_int, vp, vp, vp]
        L.orc_count_coloring.argtypes = [vp, vp, i32, vp, vp, ctypes.c_int, vp]
        L.orc_count_coloring.restype = ctypes.c_double
        L.orc_count_coloring_state.argtypes = [vp, vp, i32, vp, vp, ctypes.c_int, vp, vp]
        L.orc_count_coloring_state.restype = ctypes.c_double
        L.orc_sub_table.argtypes = [vp, vp, i32, vp, vp, ctypes.c_int, vp]
        L.orc_sub_table.restype = ctypes.c_int
        L.orc_estimate.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_estimate.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def glibc_rand(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.int32)
    lib().orc_glibc_rand(seed & 0xFFFFFFFF, n, _p(out))
    return out


def colors(seed: int, V: int, k: int) -> np.ndarray:
    out = np.zeros(V, np.int32)
    lib().orc_color(seed & 0xFFFFFFFF, V, k, _p(out))
    return out


def csc_build(V: int, src: np.ndarray, dst: np.ndarray):
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    E = len(src)
    col = np.zeros(V + 1, np.int32)
    row = np.zeros(2 * E, np.int32)
    deg = np.zeros(V, np.int32)
    rc = lib().orc_csc_build(V, E, _p(src), _p(dst), _p(col), _p(row), _p(deg))
    if rc != 0:
        raise ValueError("edge endpoint out of range")
    return col, row, deg


@dataclass
class SubInfo:
    size: int
    main: int
    aux: int
    parent: int
    L: int
    S: int
    c2c: np.ndarray = field(repr=False)
    msplit: np.ndarray = field(repr=False)   # [L][S]
    asplit: np.ndarray = field(repr=False)   # [L][S]


class Plan:
    """DivideTemplates + IndexSys restated (sg_oracle.c)."""

    def __init__(self, n: int, edges, automorphisms: bool = False):
        src = np.array([e[0] for e in edges], np.int32)
        dst = np.array([e[1] for e in edges], np.int32)
        self._h = lib().orc_plan_create(n, len(edges), _p(src), _p(dst), 1 if automorphisms else 0)
        if not self._h:
            raise ValueError("template must be a tree with 1 < n <= 32 vertices")
        self.k = lib().orc_plan_k(self._h)
        self.nsub = lib().orc_plan_nsub(self._h)
        self.aut = lib().orc_plan_aut(self._h)
        self.subs = []
        for s in range(self.nsub):
            info = np.zeros(6, np.int32)
            lib().orc_plan_sub(self._h, s, _p(info))
            size, m, a, par, L, S = (int(x) for x in info)
            c2c = np.zeros(L, np.int32)
            ms = np.zeros(max(L * S, 1), np.int32)
            as_ = np.zeros(max(L * S, 1), np.int32)
            lib().orc_plan_tables(self._h, s, _p(c2c), _p(ms), _p(as_))
            self.subs.append(SubInfo(size, m, a, par, L, S, c2c,
                                     ms[: L * S].reshape(L, S), as_[: L * S].reshape(L, S)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_plan_destroy(h)
            self._h = None


MODE_REF = 0       # FP32 tables, reference arithmetic (isPruned=1)
MODE_FP64 = 1      # FP64 tables, no scaling
MODE_ORIGINAL = 2  # isPruned=0 on a CSC graph: the SpMV buffer accumulates (state carried)
MODE_ORIGINAL_CSR = 3  # isPruned=0 on a CSR graph: a fresh aggregation per split


def count_coloring(col: np.ndarray, row: np.ndarray, plan: Plan, color: np.ndarray,
                   mode: int = MODE_REF, want_root: bool = False, state: np.ndarray | None = None):
    """One coloring's raw count.  Mode 2 starts from `state` (float32 [V], the
    CountMat's SpMV buffer, updated in place) or from zeros."""
    V = len(col) - 1
    col = np.ascontiguousarray(col, np.int32)
    row = np.ascontiguousarray(row, np.int32)
    color = np.ascontiguousarray(color, np.int32)
    root = np.zeros(V, np.float64) if want_root else None
    if state is not None:
        assert state.dtype == np.float32 and state.flags.c_contiguous and len(state) == V
    r = lib().orc_count_coloring_state(_p(col), _p(row), V, plan._h, _p(color), mode,
                                       _p(state) if state is not None else None, _p(root) if want_root else None)
    return (r, root) if want_root else r


def count_colorings(col: np.ndarray, row: np.ndarray, plan: Plan, colors, mode: int = MODE_REF) -> np.ndarray:
    """Raw counts of several colorings run one after another on one CountMat
    (mode 2 carries its SpMV buffer from each coloring to the next)."""
    V = len(col) - 1
    state = np.zeros(V, np.float32) if mode == MODE_ORIGINAL else None
    return np.array([count_coloring(col, row, plan, c, mode, state=state) for c in colors])


def sub_table(col, row, plan: Plan, color, s: int) -> np.ndarray:
    """Column-major [L][V] FP32 table of sub s (reference arithmetic)."""
    V = len(col) - 1
    L = plan.subs[s].L
    out = np.zeros(L * V, np.float32)
    rc = lib().orc_sub_table(_p(np.ascontiguousarray(col, np.int32)), _p(np.ascontiguousarray(row, np.int32)),
                             V, plan._h, _p(np.ascontiguousarray(color, np.int32)), s, _p(out))
    if rc:
        raise ValueError("bad sub index")
    return out.reshape(L, V)


def estimate(raw, k: int, aut: int = 1) -> float:
    raw = np.ascontiguousarray(raw, np.float64)
    return lib().orc_estimate(_p(raw), len(raw), k, aut)


# --------------------------------------------------------------------------
# compiled-reference dumps (oracle/_ref/ref_oracle)
# --------------------------------------------------------------------------
def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "ref_oracle"))


def run_ref(graph_txt: str, template: str, ncol: int, seed: int, outdir: str, threads: int = 4,
            dump_tables: bool = False, automorphisms: bool = False, is_pruned: int = 1, use_spmm: int = 1,
            csr: bool = False, light: bool = False) -> dict:
    """Runs the compiled reference's CountMat (oracle/_ref/ref_oracle) and
    loads what it wrote: colorings seeded srand(seed + c) on one thread, the
    counting loops on `threads` threads, with the isPruned / useSPMM flags of
    CountMat::initialization and a CSRGraph instead of the CSCGraph when
    csr=True.  light=True writes only the raw counts and per-coloring times."""
    exe = os.path.join(REF_DIR, "ref_oracle")
    subprocess.check_call([exe, graph_txt, template, str(ncol), str(seed), str(threads), outdir,
                           "1" if dump_tables else "0", "1" if automorphisms else "0", str(is_pruned),
                           str(use_spmm), "1" if csr else "0", "1" if light else "0"],
                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                          env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
    return load_ref_dump(outdir)


def load_ref_dump(d: str) -> dict:
    out: dict = {}
    out["raw"] = np.array([float(x) for x in open(os.path.join(d, "raw.txt")).read().split()])
    tp = os.path.join(d, "times.txt")
    if os.path.exists(tp):
        out["times"] = np.array([float(x) for x in open(tp).read().split()])
    out["aut"] = int(open(os.path.join(d, "aut.txt")).read())
    pre = "csc" if os.path.exists(os.path.join(d, "csc_col.i32")) else "csr"
    if not os.path.exists(os.path.join(d, f"{pre}_col.i32")):
        return out   # light run
    if pre == "csc":
        col = np.fromfile(os.path.join(d, "csc_col.i32"), np.int32)
        out["col"] = col
        out["row"] = np.fromfile(os.path.join(d, "csc_row.i32"), np.int32)
        V = len(col) - 1
    else:
        out["csr_row"] = np.fromfile(os.path.join(d, "csr_row.i32"), np.int32)
        out["csr_col"] = np.fromfile(os.path.join(d, "csr_col.i32"), np.int32)
        V = len(out["csr_row"]) - 1
    out["V"] = V
    c = np.fromfile(os.path.join(d, "colors.i32"), np.int32)
    out["colors"] = c.reshape(-1, V) if V else c
    subs = []
    with open(os.path.join(d, "plan.txt")) as f:
        lines = f.read().splitlines()
    hdr = lines[0].split()
    out["k"] = int(hdr[1])
    i = 1
    while i < len(lines):
        t = lines[i].split()
        assert t[0] == "sub"
        s = dict(size=int(t[3]), main=int(t[5]), aux=int(t[7]), parent=int(t[9]), L=int(t[11]), S=int(t[13]))
        i += 1
        s["c2c"] = np.array(lines[i].split()[1:], np.int32)
        i += 1
        if s["size"] > 1:
            s["msplit"] = np.array(lines[i].split()[1:], np.int32).reshape(s["L"], s["S"])
            s["asplit"] = np.array(lines[i + 1].split()[1:], np.int32).reshape(s["L"], s["S"])
            i += 2
        subs.append(s)
    out["subs"] = subs
    tdir = os.path.join(d, "tables")
    tables = {}
    if os.path.isdir(tdir):
        for fn in os.listdir(tdir):
            s = int(fn[1:].split(".")[0])
            tables[s] = np.fromfile(os.path.join(tdir, fn), np.float32).reshape(subs[s]["L"], V)
    out["tables"] = tables
    rd = os.path.join(d, "raw_dump.txt")
    if os.path.exists(rd):
        out["raw_dump"] = float(open(rd).read())
    return out
