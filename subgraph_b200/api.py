"""Host-side mirror of the reference's interfaces for the counting path.

Class and method names follow dsc-nec/subgraph so code written against the
reference reads the same:
  EdgeList          EdgeList.hpp:19-66
  CSCGraph          CSCGraph.hpp:22-90 (createFromEdgeListFile, serialize, deserialize)
  CSRGraph          CSRGraph.hpp:20-146
  Graph             Graph.hpp:11-66 (the template: read_enlist)
  DivideTemplates   DivideTemplates.hpp:13-64
  IndexSys          IndexSys.hpp:10-90
  CountMat          CountMat.hpp:19-191 (initialization, compute)
Everything here forwards to libsubgraph_b200.so through the C ABI; the
counting itself runs in the library's sm_100a kernels.
"""
from __future__ import annotations

import ctypes
import time
from typing import Iterable, Optional, Sequence

import numpy as np

from ._lib import (MODE_FP64, MODE_ORIGINAL, MODE_ORIGINAL_CSR, MODE_REFERENCE, CountOpts, CountStats, SGError, check, lib)

DUMMY_VAL = 93620


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _take(ptr: ctypes.c_void_p, n: int, dtype=np.int32) -> np.ndarray:
    """Copies a library-allocated array into numpy and frees it."""
    if n == 0:
        lib().sg_free(ptr)
        return np.zeros(0, dtype)
    buf = (ctypes.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr.value)
    out = np.frombuffer(buf, dtype=dtype).copy()
    lib().sg_free(ptr)
    return out


# ---------------------------------------------------------------------------
class EdgeList:
    """Text edge list "V\\nE\\nu v\\n..." (EdgeList.cpp:34-116, hole removal included)."""

    def __init__(self, fileName: Optional[str] = None, V: int = 0, src=None, dst=None):
        if fileName is not None:
            v, e = ctypes.c_int32(), ctypes.c_int64()
            ps, pd = ctypes.c_void_p(), ctypes.c_void_p()
            check(lib().sg_edgelist_read(fileName.encode(), ctypes.byref(v), ctypes.byref(e),
                                         ctypes.byref(ps), ctypes.byref(pd)))
            self._V = v.value
            self._src = _take(ps, e.value)
            self._dst = _take(pd, e.value)
        else:
            self._V = int(V)
            self._src = np.ascontiguousarray(src, np.int32)
            self._dst = np.ascontiguousarray(dst, np.int32)

    def getNumVertices(self) -> int:
        return self._V

    def getNumEdges(self) -> int:
        return len(self._src)

    def getSrcList(self) -> np.ndarray:
        return self._src

    def getDstList(self) -> np.ndarray:
        return self._dst

    def write(self, path: str) -> None:
        check(lib().sg_edgelist_write(path.encode(), self._V, len(self._src), _p(self._src), _p(self._dst)))


def rmat(scale: int, edge_factor: int, seed: int = 1, a: float = 0.57, b: float = 0.19, c: float = 0.19) -> EdgeList:
    """Seeded R-MAT graph: symmetrised, self loops and duplicates removed."""
    v, e = ctypes.c_int32(), ctypes.c_int64()
    ps, pd = ctypes.c_void_p(), ctypes.c_void_p()
    check(lib().sg_rmat_generate(scale, edge_factor, a, b, c, seed, ctypes.byref(v), ctypes.byref(e),
                                 ctypes.byref(ps), ctypes.byref(pd)))
    return EdgeList(V=v.value, src=_take(ps, e.value), dst=_take(pd, e.value))


# ---------------------------------------------------------------------------
class _DeviceAdjacency:
    """A device copy of an adjacency (offsets + neighbours in summation order)."""

    def __init__(self):
        self._dev = None
        self._dev_device = None

    def _arrays(self):
        raise NotImplementedError

    def device_graph(self, device: int = 0) -> "DeviceGraph":
        if self._dev is None or self._dev_device != device:
            off, nbr = self._arrays()
            self._dev = DeviceGraph(off, nbr, device)
            self._dev_device = device
        return self._dev


class CSCGraph(_DeviceAdjacency):
    """CSCGraph<int32_t, float> (CSCGraph.hpp:22-90)."""

    def __init__(self):
        super().__init__()
        self._V = 0
        self._numEdges = 0
        self._indexCol = np.zeros(1, np.int32)
        self._indexRow = np.zeros(0, np.int32)
        self._degList = np.zeros(0, np.int32)

    def createFromEdgeListFile(self, numVerts: int, numEdges: int, srcList, dstList, isBenchmark: bool = False):
        src = np.ascontiguousarray(srcList, np.int32)
        dst = np.ascontiguousarray(dstList, np.int32)
        if len(src) != numEdges or len(dst) != numEdges:
            raise ValueError("numEdges does not match the edge arrays")
        pc, pr, pd = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().sg_csc_build(numVerts, numEdges, _p(src), _p(dst), ctypes.byref(pc), ctypes.byref(pr),
                                 ctypes.byref(pd)))
        self._V = int(numVerts)
        self._numEdges = int(numEdges)
        self._indexCol = _take(pc, self._V + 1)
        self._indexRow = _take(pr, int(self._indexCol[-1]))
        self._degList = _take(pd, self._V)
        self._dev = None

    def splitCSC(self, numsplits: int) -> None:
        """The reference's row-owner split for its OpenMP SpMM (CSCGraph.hpp:180-217); the
        device kernels balance work by degree order instead, so this only validates."""
        if numsplits < 1:
            raise ValueError("numsplits must be >= 1")

    def serialize(self, path: str) -> None:
        check(lib().sg_graph_data_write(path.encode(), self._V, self._numEdges, _p(self._indexCol),
                                        _p(self._indexRow), _p(self._degList)))

    def deserialize(self, path: str) -> None:
        v, ne = ctypes.c_int32(), ctypes.c_int32()
        pc, pr, pd = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().sg_graph_data_read(path.encode(), ctypes.byref(v), ctypes.byref(ne), ctypes.byref(pc),
                                       ctypes.byref(pr), ctypes.byref(pd)))
        self._V, self._numEdges = v.value, ne.value
        self._indexCol = _take(pc, self._V + 1)
        self._indexRow = _take(pr, int(self._indexCol[-1]))
        self._degList = _take(pd, self._V)
        self._dev = None

    def getNumVertices(self) -> int:
        return self._V

    def getNNZ(self) -> int:
        return int(self._indexCol[-1])

    def getIndexCol(self) -> np.ndarray:
        return self._indexCol

    def getIndexRow(self) -> np.ndarray:
        return self._indexRow

    def getDegList(self) -> np.ndarray:
        return self._degList

    def getColLen(self, colId: int) -> int:
        return int(self._indexCol[colId + 1] - self._indexCol[colId])

    def _arrays(self):
        return self._indexCol, self._indexRow


class CSRGraph(_DeviceAdjacency):
    """CSRGraph (CSRGraph.hpp:20-146): neighbours in insertion order."""

    def __init__(self):
        super().__init__()
        self._V = 0
        self._numEdges = 0
        self._indexRow = np.zeros(1, np.int32)
        self._indexCol = np.zeros(0, np.int32)
        self._degList = np.zeros(0, np.int32)

    def createFromEdgeListFile(self, numVerts: int, numEdges: int, srcList, dstList, useMKL: bool = False,
                               useRcm: bool = False, isBenchmark: bool = False):
        src = np.ascontiguousarray(srcList, np.int32)
        dst = np.ascontiguousarray(dstList, np.int32)
        pr, pc, pd = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().sg_csr_build(numVerts, numEdges, _p(src), _p(dst), ctypes.byref(pr), ctypes.byref(pc),
                                 ctypes.byref(pd)))
        self._V = int(numVerts)
        self._numEdges = int(numEdges)
        self._indexRow = _take(pr, self._V + 1)
        self._indexCol = _take(pc, int(self._indexRow[-1]))
        self._degList = _take(pd, self._V)
        self._dev = None

    def getNumVertices(self) -> int:
        return self._V

    def getNNZ(self) -> int:
        return int(self._indexRow[-1])

    def getIndexRow(self) -> np.ndarray:
        return self._indexRow

    def getIndexCol(self) -> np.ndarray:
        return self._indexCol

    def getDegList(self) -> np.ndarray:
        return self._degList

    def useMKL(self) -> bool:
        return False

    def _arrays(self):
        return self._indexRow, self._indexCol


class DeviceGraph:
    """sg_graph: an adjacency resident on one GPU."""

    def __init__(self, offsets: np.ndarray, neighbors: np.ndarray, device: int = 0):
        off = np.ascontiguousarray(offsets, np.int32)
        nbr = np.ascontiguousarray(neighbors, np.int32)
        h = ctypes.c_void_p()
        check(lib().sg_graph_create(_p(off), _p(nbr), len(off) - 1, len(nbr), device, ctypes.byref(h)))
        self._h = h
        self.V = len(off) - 1
        self.nnz = len(nbr)

    @classmethod
    def _wrap(cls, h):
        self = cls.__new__(cls)
        self._h = h
        V, nnz = ctypes.c_int32(), ctypes.c_int64()
        check(lib().sg_graph_info(h, ctypes.byref(V), ctypes.byref(nnz), None))
        self.V, self.nnz = V.value, nnz.value
        return self

    @classmethod
    def from_edges(cls, V: int, src, dst, device: int = 0) -> "DeviceGraph":
        """CSC of the symmetrised edge list built on the GPU (CSCGraph::createFromEdgeListFile)."""
        s = np.ascontiguousarray(src, np.int32)
        d = np.ascontiguousarray(dst, np.int32)
        if len(s) != len(d):
            raise ValueError("src and dst differ in length")
        h = ctypes.c_void_p()
        check(lib().sg_graph_create_edges(V, _p(s), _p(d), len(s), device, ctypes.byref(h)))
        return cls._wrap(h)

    @classmethod
    def from_edge_list_file(cls, path: str, device: int = 0) -> "DeviceGraph":
        """An edge-list text file ("V\\nE\\nu v\\n...") parsed and built on the GPU."""
        h = ctypes.c_void_p()
        check(lib().sg_graph_create_text(path.encode(), device, ctypes.byref(h)))
        return cls._wrap(h)

    @classmethod
    def from_rmat(cls, scale: int, edge_factor: int, a: float = 0.57, b: float = 0.19, c: float = 0.19,
                  seed: int = 1, device: int = 0) -> "DeviceGraph":
        """An R-MAT graph generated, deduplicated and built on the GPU."""
        h = ctypes.c_void_p()
        check(lib().sg_graph_create_rmat(scale, edge_factor, a, b, c, seed & 0xFFFFFFFFFFFFFFFF, device,
                                         ctypes.byref(h)))
        return cls._wrap(h)

    def csc(self):
        """(offsets, neighbors) of the graph in original vertex order."""
        off = np.zeros(self.V + 1, np.int32)
        nbr = np.zeros(max(self.nnz, 1), np.int32)
        check(lib().sg_graph_download_csc(self._h, _p(off), _p(nbr)))
        return off, nbr[: self.nnz]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().sg_graph_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def max_degree(self) -> int:
        md = ctypes.c_int32()
        check(lib().sg_graph_info(self._h, None, None, ctypes.byref(md)))
        return md.value

    def colors(self, k: int, seed: int) -> np.ndarray:
        out = np.zeros(self.V, np.int32)
        check(lib().sg_colors(self._h, k, seed & 0xFFFFFFFF, _p(out)))
        return out


# ---------------------------------------------------------------------------
class Graph:
    """A tree template (Graph.hpp:11-66)."""

    def __init__(self, n: int = 0, edges: Sequence[tuple[int, int]] = ()):
        self._plan = None
        self.n = 0
        self.edges: list[tuple[int, int]] = []
        if n:
            self.build_graph(n, edges)

    def read_enlist(self, file_name: str) -> None:
        h = ctypes.c_void_p()
        check(lib().sg_plan_read(file_name.encode(), ctypes.byref(h)))
        self._set_plan(h)

    def build_graph(self, n: int, edges: Iterable[tuple[int, int]]) -> None:
        edges = [tuple(map(int, e)) for e in edges]
        src = np.array([e[0] for e in edges], np.int32)
        dst = np.array([e[1] for e in edges], np.int32)
        h = ctypes.c_void_p()
        check(lib().sg_plan_create(n, len(edges), _p(src), _p(dst), ctypes.byref(h)))
        self._set_plan(h)

    def _set_plan(self, h):
        if self._plan is not None:
            lib().sg_plan_destroy(self._plan)
        self._plan = h
        k = ctypes.c_int32()
        check(lib().sg_plan_info(h, ctypes.byref(k), None, None, None))
        self.n = k.value
        n2 = ctypes.c_int32()
        src = np.zeros(64, np.int32)
        dst = np.zeros(64, np.int32)
        check(lib().sg_plan_sub_edges(h, 0, ctypes.byref(n2), _p(src), _p(dst)))
        self.edges = [(int(a), int(b)) for a, b in zip(src[: self.n - 1], dst[: self.n - 1])]

    def __del__(self):
        if getattr(self, "_plan", None) is not None:
            lib().sg_plan_destroy(self._plan)
            self._plan = None

    def get_vert_num(self) -> int:
        return self.n

    def get_edge_num(self) -> int:
        return 2 * len(self.edges)

    @property
    def plan(self):
        if self._plan is None:
            raise ValueError("template not loaded")
        return self._plan

    def automorphisms(self) -> int:
        c = ctypes.c_int32()
        check(lib().sg_plan_automorphisms(self.plan, ctypes.byref(c)))
        return c.value

    def shared_tables(self) -> list[int]:
        """Per sub: the sub processed before it whose table it reuses, or -1."""
        k, ns = ctypes.c_int32(), ctypes.c_int32()
        check(lib().sg_plan_info(self.plan, ctypes.byref(k), ctypes.byref(ns), None, None))
        out = np.zeros(ns.value, np.int32)
        check(lib().sg_plan_shared_tables(self.plan, _p(out)))
        return [int(x) for x in out]


class DivideTemplates:
    """Sub-template chain of a template (DivideTemplates.hpp:13-64)."""

    def __init__(self):
        self._g: Optional[Graph] = None
        self._info: list[np.ndarray] = []

    def DivideTp(self, tp: Graph) -> None:
        self._g = tp
        k, ns = ctypes.c_int32(), ctypes.c_int32()
        check(lib().sg_plan_info(tp.plan, ctypes.byref(k), ctypes.byref(ns), None, None))
        self._info = []
        for s in range(ns.value):
            info = np.zeros(7, np.int32)
            check(lib().sg_plan_sub(tp.plan, s, _p(info)))
            self._info.append(info)

    def sort_tps(self) -> None:
        """The plan is created in the sorted order already."""

    def get_subtps_num(self) -> int:
        return len(self._info)

    def get_main_node_idx(self, s: int) -> int:
        return int(self._info[s][1])

    def get_aux_node_idx(self, s: int) -> int:
        return int(self._info[s][2])

    def get_parent(self, s: int) -> int:
        return int(self._info[s][3])

    def get_sub_size(self, s: int) -> int:
        return int(self._info[s][0])

    def get_main_node_vert_num(self, s: int) -> int:
        return self.get_sub_size(self.get_main_node_idx(s))

    def get_aux_node_vert_num(self, s: int) -> int:
        return self.get_sub_size(self.get_aux_node_idx(s))

    def get_subtp_edges(self, s: int) -> tuple[int, list[tuple[int, int]]]:
        n = ctypes.c_int32()
        src = np.zeros(64, np.int32)
        dst = np.zeros(64, np.int32)
        check(lib().sg_plan_sub_edges(self._g.plan, s, ctypes.byref(n), _p(src), _p(dst)))
        return n.value, [(int(a), int(b)) for a, b in zip(src[: n.value - 1], dst[: n.value - 1])]


class IndexSys:
    """Color-set index tables (IndexSys.hpp:10-90)."""

    def __init__(self):
        self._g: Optional[Graph] = None

    def initialization(self, color_num: int, sub_len: int, sub_tps: Graph, divider: DivideTemplates) -> None:
        if sub_tps.get_vert_num() != color_num:
            raise ValueError("color_num must equal the template size")
        self._g = sub_tps

    def getCombToCountTable(self, s: int) -> np.ndarray:
        return self.tables(s)[0]

    def getSplitToCountTable(self, s: int) -> tuple[np.ndarray, np.ndarray]:
        _, m, a = self.tables(s)
        return m, a

    def tables(self, s: int):
        info = np.zeros(7, np.int32)
        check(lib().sg_plan_sub(self._g.plan, s, _p(info)))
        L, S = int(info[4]), int(info[5])
        c2c = np.zeros(L, np.int32)
        ms = np.zeros(max(L * S, 1), np.int32)
        as_ = np.zeros(max(L * S, 1), np.int32)
        check(lib().sg_plan_tables(self._g.plan, s, _p(c2c), _p(ms), _p(as_)))
        return c2c, ms[: L * S].reshape(L, S), as_[: L * S].reshape(L, S)

    @staticmethod
    def comb_calc(n: int, k: int) -> int:
        from math import comb
        return comb(n, k) if 0 <= k <= n else 0


# ---------------------------------------------------------------------------
def count(graph: DeviceGraph, template: Graph, n_colorings: int = 1, seed_base: int = 0,
          mode: int = MODE_REFERENCE, batch: int = 0, hub_threshold: int = 1024,
          return_stats: bool = False, profile: bool = False, autotune: bool = True, exact: bool = False,
          wait_limit_ms: int = 0, blocked: bool = True, persistent: bool = False, rooted: bool = True,
          flat: bool = True):
    """Raw colorful counts of n_colorings colorings (coloring c uses srand(seed_base + c))."""
    o = CountOpts()
    lib().sg_count_opts_default(ctypes.byref(o))
    o.n_colorings = n_colorings
    o.seed_base = seed_base & 0xFFFFFFFF
    o.mode = mode
    o.batch = batch
    o.hub_threshold = hub_threshold
    o.profile = 1 if profile else 0
    o.no_autotune = 0 if autotune else 1
    o.exact = 1 if exact else 0
    o.wait_limit_ms = wait_limit_ms
    o.no_blocked = 0 if blocked else 1
    o.no_rooted = 0 if rooted else 1
    o.no_flat = 0 if flat else 1
    o.persistent = 1 if persistent else 0
    raw = np.zeros(n_colorings, np.float64)
    st = CountStats()
    check(lib().sg_count(graph.handle, template.plan, ctypes.byref(o), _p(raw), ctypes.byref(st)))
    if return_stats:
        return raw, {k: getattr(st, k) for k, _ in CountStats._fields_}
    return raw


def debug_count_unsatisfiable_wait(graph: DeviceGraph, template: Graph, n_colorings: int, seed_base: int,
                                   batch: int, wait_limit_ms: int):
    """Test of the bounded waits: the persistent batched form with one dependency
    that nothing satisfies.  Raises SGError (status 4, timeout) when the waits
    give up as they must."""
    o = CountOpts()
    lib().sg_count_opts_default(ctypes.byref(o))
    o.n_colorings = n_colorings
    o.seed_base = seed_base & 0xFFFFFFFF
    o.batch = batch
    o.wait_limit_ms = wait_limit_ms
    raw = np.zeros(n_colorings, np.float64)
    check(lib().sg_debug_count_unsatisfiable_wait(graph.handle, template.plan, ctypes.byref(o), _p(raw)))
    return raw


def count_jobs(graph: DeviceGraph, templates, seeds, mode: int = MODE_REFERENCE, hub_threshold: int = 1024,
               exact: bool = False, wait_limit_ms: int = 0, return_latency: bool = False, return_stats: bool = False,
               persistent: bool = False, streams: int = 0):
    """One coloring each of jobs with different templates on one graph (job j:
    templates[j] seeded srand(seeds[j])): their stage launches spread over
    `streams` CUDA streams (0: 8), or with persistent=True in persistent
    work-queue launches.  Returns the raw counts; with return_latency also each
    job's latency (ms)."""
    n = len(templates)
    if n != len(seeds):
        raise ValueError("one seed per job")
    plans = (ctypes.c_void_p * n)(*[t.plan for t in templates])
    sd = np.ascontiguousarray([int(x) & 0xFFFFFFFF for x in seeds], np.uint32)
    o = CountOpts()
    lib().sg_count_opts_default(ctypes.byref(o))
    o.mode = mode
    o.hub_threshold = hub_threshold
    o.exact = 1 if exact else 0
    o.wait_limit_ms = wait_limit_ms
    o.persistent = 1 if persistent else 0
    o.batch = streams
    raw = np.zeros(n, np.float64)
    lat = np.zeros(n, np.float64)
    st = CountStats()
    check(lib().sg_count_jobs(graph.handle, n, ctypes.cast(plans, ctypes.c_void_p), _p(sd), ctypes.byref(o), _p(raw),
                              _p(lat), ctypes.byref(st)))
    out = [raw]
    if return_latency:
        out.append(lat)
    if return_stats:
        out.append({k: getattr(st, k) for k, _ in CountStats._fields_})
    return out[0] if len(out) == 1 else tuple(out)


def estimate(raw: Sequence[float], k: int, automorphisms: int = 1) -> float:
    r = np.ascontiguousarray(raw, np.float64)
    out = ctypes.c_double()
    check(lib().sg_estimate(_p(r), len(r), k, automorphisms, ctypes.byref(out)))
    return out.value


def debug_sub_table(graph: DeviceGraph, template: Graph, seed: int, s: int, mode: int = MODE_REFERENCE,
                    hub_threshold: int = 0) -> np.ndarray:
    info = np.zeros(7, np.int32)
    check(lib().sg_plan_sub(template.plan, s, _p(info)))
    L = int(info[4])
    out = np.zeros(L * graph.V, np.float64 if mode == MODE_FP64 else np.float32)
    check(lib().sg_debug_sub_table(graph.handle, template.plan, seed & 0xFFFFFFFF, mode, hub_threshold, s, _p(out)))
    return out.reshape(L, graph.V)


def debug_root(graph: DeviceGraph, template: Graph, seed: int, mode: int = MODE_REFERENCE,
               hub_threshold: int = 0):
    root = np.zeros(graph.V, np.float64)
    raw = ctypes.c_double()
    check(lib().sg_debug_root(graph.handle, template.plan, seed & 0xFFFFFFFF, mode, hub_threshold, _p(root),
                              ctypes.byref(raw)))
    return root, raw.value


class CountMat:
    """The counting engine (CountMat.hpp:19-191)."""

    def __init__(self):
        h = ctypes.c_void_p()
        check(lib().sg_countmat_create(ctypes.byref(h)))
        self._h = h
        self._graph_ref = None
        self._itr = 1

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().sg_countmat_destroy(h)
            self._h = None

    def initialization(self, graph: Optional[CSRGraph], graphCSC: Optional[CSCGraph], thd_num: int, itr_num: int,
                       isPruned: int = 1, useSPMM: int = 1, vtuneStart: int = -1,
                       calculate_automorphisms: bool = False, device: int = 0) -> None:
        if (graph is None) == (graphCSC is None):
            raise ValueError("exactly one of graph (CSR) and graphCSC must be given")
        src = graph if graph is not None else graphCSC
        dg = src.device_graph(device)
        self._graph_ref = dg
        check(lib().sg_countmat_initialization(self._h, dg.handle if graph is not None else None,
                                               dg.handle if graphCSC is not None else None, thd_num, itr_num,
                                               isPruned, useSPMM, vtuneStart, 1 if calculate_automorphisms else 0))
        self._itr = itr_num

    def set_seed(self, seed_base: int) -> None:
        check(lib().sg_countmat_set_seed(self._h, seed_base & 0xFFFFFFFF))

    def compute(self, templates: Graph, isEstimate: bool = False, verbose: bool = False) -> float:
        out = ctypes.c_double()
        check(lib().sg_countmat_compute(self._h, templates.plan, 1 if isEstimate else 0, 1 if verbose else 0,
                                        ctypes.byref(out)))
        return out.value

    def raw_counts(self) -> np.ndarray:
        r = np.zeros(self._itr, np.float64)
        check(lib().sg_countmat_raw(self._h, _p(r)))
        return r


__all__ = ["EdgeList", "CSCGraph", "CSRGraph", "DeviceGraph", "Graph", "DivideTemplates", "IndexSys", "CountMat",
           "count", "count_jobs", "estimate", "rmat", "debug_sub_table", "debug_root", "MODE_REFERENCE", "MODE_FP64",
           "MODE_ORIGINAL", "MODE_ORIGINAL_CSR", "DUMMY_VAL", "SGError"]
