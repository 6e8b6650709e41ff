"""Parity of the sm_100a path (through the C ABI) with the reference and the oracle.

Bars:
  * colors, CSC-derived tables and split enumeration: bit-exact;
  * exact mode (every neighbour list summed in order, products rounded then
    added as the reference does):
    every sub-template table bit-identical to the reference's, per-vertex
    root values identical, raw counts equal up to the final FP64 sum
    (relative 1e-12);
  * default mode (chunked hub aggregation, fused multiply-add in the packed
    eMA): raw counts within 1e-5 relative of the reference, estimates within
    1e-6;
  * FP64 mode: within 1e-12 of the oracle's FP64 tables.
"""
import random

import numpy as np
import pytest

import subgraph_b200 as sg
from oracle import oracle as O
from tests.helpers import TEMPLATES, prufer_tree, rel, sha

pytestmark = pytest.mark.gpu

_graphs = {}


def dev_graph(golden, name):
    if name not in _graphs:
        _, _, _, col, row = golden.graph(name)
        _graphs[name] = (sg.DeviceGraph(col, row), col, row)
    return _graphs[name]


@pytest.mark.parametrize("V", [1, 1000, 1024, 1025, 5000, 70001])
def test_colors_bit_exact(V):
    off = np.zeros(V + 1, np.int32)
    g = sg.DeviceGraph(off, np.zeros(0, np.int32))
    for k in (2, 3, 5, 12, 16):
        for seed in (0, 7, 2**31 + 3):
            assert np.array_equal(g.colors(k, seed), O.colors(seed, V, k)), (V, k, seed)


def test_golden_colors(golden):
    for c in golden.cases:
        g, _, _ = dev_graph(golden, c.graph)
        for i in range(c.ncol):
            assert np.array_equal(g.colors(c.n, c.seed + i), c.colors[i]), (c.key, i)


def test_golden_tables_bit_exact(golden):
    n = 0
    for c in golden.cases:
        if not c.table_sha:
            continue
        g, _, _ = dev_graph(golden, c.graph)
        t = sg.Graph(c.n, c.edges)
        for s, digest in c.table_sha.items():
            T = sg.debug_sub_table(g, t, c.seed, s, hub_threshold=0)
            assert sha(T) == digest, (c.key, s)
            n += 1
    assert n > 30


def test_golden_raw_counts_exact_mode(golden):
    for c in golden.cases:
        g, col, row = dev_graph(golden, c.graph)
        t = sg.Graph(c.n, c.edges)
        raw = sg.count(g, t, c.ncol, c.seed, exact=True)
        for i in range(c.ncol):
            assert rel(raw[i], c.raw[i]) <= 1e-12, (c.key, i, raw[i], c.raw[i])
        # per-vertex root values are the reference's bufLastSub; summed in vertex order they
        # give the reference's count to the last bit
        root, raw_seq = sg.debug_root(g, t, c.seed, hub_threshold=0)
        assert raw_seq == c.raw[0], (c.key, raw_seq, c.raw[0])
        P = O.Plan(c.n, c.edges)
        _, root_oracle = O.count_coloring(col, row, P, c.colors[0], want_root=True)
        assert np.array_equal(root, root_oracle), c.key


def test_golden_tables_bit_exact_through_hub_kernel(golden):
    """Vertices above the hub threshold (8 here: most rmat vertices) aggregated by
    the exact-order hub kernel (columns split among lanes, every neighbour list
    summed in order): every table still bit-identical to the reference's."""
    n = 0
    for c in golden.cases:
        if not c.table_sha:
            continue
        g, _, _ = dev_graph(golden, c.graph)
        t = sg.Graph(c.n, c.edges)
        for s, digest in c.table_sha.items():
            T = sg.debug_sub_table(g, t, c.seed, s, hub_threshold=8)
            assert sha(T) == digest, (c.key, s)
            n += 1
    assert n > 30


def test_golden_raw_counts_hub_mode(golden):
    """The default (fast) path with a hub threshold of 8: exact-order hubs, so the
    counts are the reference's up to fused multiply-adds in the packed eMA."""
    for c in golden.cases:
        g, _, _ = dev_graph(golden, c.graph)
        t = sg.Graph(c.n, c.edges)
        raw = sg.count(g, t, c.ncol, c.seed, hub_threshold=8)
        for i in range(c.ncol):
            assert rel(raw[i], c.raw[i]) <= 1e-6, (c.key, i)
        raw = sg.count(g, t, c.ncol, c.seed, hub_threshold=8, exact=True)
        for i in range(c.ncol):
            assert rel(raw[i], c.raw[i]) <= 1e-12, (c.key, i)
        est = sg.estimate(raw, c.n)
        ref_est = O.estimate(c.raw, c.n, 1)
        assert rel(est, ref_est) <= 1e-6 or abs(est - ref_est) <= 1.0, (c.key, est, ref_est)


def test_chunked_hubs_of_the_persistent_queue(golden):
    """The persistent queue sums hub neighbour lists in chunks (another order):
    within 1e-5 of the reference."""
    for c in golden.cases[::2]:
        g, _, _ = dev_graph(golden, c.graph)
        t = sg.Graph(c.n, c.edges)
        raw = sg.count(g, t, c.ncol, c.seed, hub_threshold=8, batch=c.ncol, persistent=True)
        for i in range(c.ncol):
            assert rel(raw[i], c.raw[i]) <= 1e-5, (c.key, i)


def test_fp64_mode_matches_oracle(golden):
    for c in golden.cases[::3]:
        g, col, row = dev_graph(golden, c.graph)
        t = sg.Graph(c.n, c.edges)
        P = O.Plan(c.n, c.edges)
        raw = sg.count(g, t, 1, c.seed, mode=sg.MODE_FP64, hub_threshold=0)
        r64 = O.count_coloring(col, row, P, c.colors[0], mode=O.MODE_FP64)
        assert rel(raw[0], r64) <= 1e-12, (c.key, raw[0], r64)


def test_original_modes_match_oracle(golden):
    """isPruned=0: per-vertex root values of one coloring (from a zero SpMV
    buffer in mode 2) identical to the oracle's, inf and NaN included."""
    for c in golden.cases[::4]:
        g, col, row = dev_graph(golden, c.graph)
        t = sg.Graph(c.n, c.edges)
        P = O.Plan(c.n, c.edges)
        for mode, omode in ((sg.MODE_ORIGINAL, O.MODE_ORIGINAL), (sg.MODE_ORIGINAL_CSR, O.MODE_ORIGINAL_CSR)):
            root, _ = sg.debug_root(g, t, c.seed, mode=mode, hub_threshold=0)
            r, root_o = O.count_coloring(col, row, P, c.colors[0], mode=omode, want_root=True)
            assert np.array_equal(root, root_o, equal_nan=True), (c.key, mode)


def test_k2_template_keeps_reference_scaling(golden):
    """A 2-vertex template has no scaled sub, yet the reference multiplies the root sum by
    1e12 (CountMat.cpp:813-822); the reference mode reproduces that, FP64 mode does not."""
    c = next(c for c in golden.cases if c.template == "p2" and c.graph == "rmat10")
    g, _, _ = dev_graph(golden, c.graph)
    t = sg.Graph(2, [(0, 1)])
    raw = sg.count(g, t, 1, c.seed, exact=True)
    raw64 = sg.count(g, t, 1, c.seed, mode=sg.MODE_FP64)
    assert rel(raw[0], c.raw[0]) <= 1e-12
    assert rel(raw[0], raw64[0] * 1e12) <= 1e-12


def test_random_trees_against_oracle():
    """Random Pruefer trees (3..10 vertices) on a fresh R-MAT graph, exact mode."""
    el = sg.rmat(11, 8, seed=5)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    g = csc.device_graph()
    rng = random.Random(17)
    for i in range(12):
        n = rng.randint(3, 10)
        edges = prufer_tree(n, rng)
        P = O.Plan(n, edges)
        colors = O.colors(50 + i, csc.getNumVertices(), n)
        r_o = O.count_coloring(csc.getIndexCol(), csc.getIndexRow(), P, colors)
        raw = sg.count(g, sg.Graph(n, edges), 1, 50 + i, exact=True)
        assert rel(raw[0], r_o) <= 1e-12, (n, edges)


def test_edge_cases():
    # no edges: every count is zero
    g = sg.DeviceGraph(np.zeros(11, np.int32), np.zeros(0, np.int32))
    assert sg.count(g, sg.Graph(*TEMPLATES["p3"]), 2, 3)[0] == 0.0
    # a single edge, and a self loop only
    g = sg.DeviceGraph(np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32))
    r = sg.count(g, sg.Graph(2, [(0, 1)]), 4, 1, mode=sg.MODE_FP64)
    cols = [O.colors(1 + i, 2, 2) for i in range(4)]
    assert r.tolist() == [2.0 if c[0] != c[1] else 0.0 for c in cols]
    # V not a multiple of the tile, isolated vertices, duplicate edges
    src = np.array([0, 0, 1, 2, 5], np.int32)
    dst = np.array([1, 1, 2, 3, 5], np.int32)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(37, 5, src, dst)
    P = O.Plan(3, TEMPLATES["p3"][1])
    g = csc.device_graph()
    for seed in range(5):
        colors = O.colors(seed, 37, 3)
        ro = O.count_coloring(csc.getIndexCol(), csc.getIndexRow(), P, colors)
        assert rel(sg.count(g, sg.Graph(*TEMPLATES["p3"]), 1, seed, exact=True)[0], ro) <= 1e-12 or ro == 0.0


def test_invalid_arguments_are_errors():
    g = sg.DeviceGraph(np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32))
    with pytest.raises(sg.SGError):
        sg.count(g, sg.Graph(*TEMPLATES["p3"]), 0, 1)
    with pytest.raises(sg.SGError):
        sg.DeviceGraph(np.array([0, 1, 2], np.int32), np.array([1, 7], np.int32))
    with pytest.raises(sg.SGError):
        sg.DeviceGraph(np.array([0, 2, 1], np.int32), np.array([1, 0], np.int32))


def _p3_exact(col, row, colors):
    """Colorful P3 rooted at an end = sum over middle vertices u of ordered pairs of
    neighbours (v, w) with c(v), c(w), c(u) pairwise distinct (k = 3)."""
    V = len(col) - 1
    deg = np.diff(col)
    owner = np.repeat(np.arange(V), deg)
    h = np.zeros((V, 3), np.int64)
    np.add.at(h, (owner, colors[row]), 1)
    tot = 0
    for c in range(3):
        a, b = [x for x in range(3) if x != c]
        sel = colors == c
        tot += int((2 * h[sel, a] * h[sel, b]).sum())
    return float(tot)


def test_full_size_p3_against_closed_form():
    """Config-1 shape (R-MAT scale 16, edge factor 16, P3): per-coloring counts against
    the closed form, FP64 mode exactly, FP32 reference mode within 1e-5."""
    el = sg.rmat(16, 16, seed=1)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    g = csc.device_graph()
    t = sg.Graph(*TEMPLATES["p3"])
    raw32 = sg.count(g, t, 3, 7)
    raw64 = sg.count(g, t, 3, 7, mode=sg.MODE_FP64)
    for i in range(3):
        exact = _p3_exact(csc.getIndexCol(), csc.getIndexRow(), O.colors(7 + i, el.getNumVertices(), 3))
        assert raw64[i] == exact
        assert rel(raw32[i], exact) <= 1e-5


def test_fp32_vs_fp64_relative_error_tree12():
    """The 12-vertex tree on R-MAT scale 14: FP32 tables vs FP64 tables within 1e-5."""
    el = sg.rmat(14, 8, seed=1)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    g = csc.device_graph()
    t = sg.Graph(*TEMPLATES["tree12"])
    raw32 = sg.count(g, t, 2, 7)
    raw64 = sg.count(g, t, 2, 7, mode=sg.MODE_FP64)
    for a, b in zip(raw32, raw64):
        assert rel(a, b) <= 1e-5


def test_deterministic_runs():
    el = sg.rmat(13, 8, seed=2)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    g = csc.device_graph()
    t = sg.Graph(*TEMPLATES["spider7"])
    a = sg.count(g, t, 3, 9, hub_threshold=16)
    b = sg.count(g, t, 3, 9, hub_threshold=16)
    assert np.array_equal(a, b)


def test_hub_rows_equal_no_hubs(golden):
    """Exact mode: the hub kernel's rows (each column summed over the whole
    neighbour list in order, a neighbour's slice copied only where the hub's
    colour and the neighbour's need it) give every vertex the values of a run
    without hub vertices, whose aggregation is all in the tiles (the counts to
    the rounding of the FP64 sum of the tile partials, whose tiles follow each
    run's tile shapes: shapes tuned earlier in the process for one of the two
    hub settings are used even without autotuning).  Repeated tuned calls are
    bit-identical."""
    for gname in ("rmat10", "rmat12"):
        _, _, _, col, row = golden.graph(gname)
        g = sg.DeviceGraph(col, row)
        for tname in ("tree12", "spider7", "tree5"):
            t = sg.Graph(*TEMPLATES[tname])
            for mode in (sg.MODE_REFERENCE, sg.MODE_FP64):
                a = sg.count(g, t, 3, 5, mode=mode, exact=True, autotune=False, hub_threshold=16)
                b = sg.count(g, t, 3, 5, mode=mode, exact=True, autotune=False, hub_threshold=0)
                assert all(rel(x, y) <= 1e-12 for x, y in zip(a, b)), (gname, tname, mode, a, b)
                c = sg.count(g, t, 3, 5, mode=mode, exact=True, hub_threshold=16)
                d = sg.count(g, t, 3, 5, mode=mode, exact=True, hub_threshold=16)
                assert np.array_equal(c, d), (gname, tname, mode, c, d)
                assert all(rel(x, y) <= 1e-12 for x, y in zip(c, b)), (gname, tname, mode, c, b)


def test_countmat_interface(golden):
    c = next(c for c in golden.cases if c.template == "tree5" and c.graph == "rmat10")
    V, s, d, _, _ = golden.graph("rmat10")
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(V, len(s), s, d)
    csc.splitCSC(16)
    t = sg.Graph(c.n, c.edges)
    cm = sg.CountMat()
    cm.initialization(None, csc, 8, c.ncol, 1, 1, -1, False)
    cm.set_seed(c.seed)
    est = cm.compute(t)
    raw = cm.raw_counts()
    assert all(rel(a, b) <= 1e-6 for a, b in zip(raw, c.raw))
    assert rel(est, O.estimate(c.raw, c.n, 1)) <= 1e-6


def test_fast_path_close_to_exact(golden):
    """The default path (packed eMA with fused products, tuned shapes) against the
    exact path on the 12-vertex tree: within 1e-6, and deterministic."""
    c = next(c for c in golden.cases if c.template == "tree12" and c.graph == "rmat12")
    g, _, _ = dev_graph(golden, c.graph)
    t = sg.Graph(c.n, c.edges)
    fast = sg.count(g, t, c.ncol, c.seed)
    fast2 = sg.count(g, t, c.ncol, c.seed)
    exact = sg.count(g, t, c.ncol, c.seed, exact=True, autotune=False)
    assert np.array_equal(fast, fast2)
    for a, b, r in zip(fast, exact, c.raw):
        assert rel(a, b) <= 1e-6 and rel(b, r) <= 1e-12


def test_csr_input_path_against_oracle():
    """CSRGraph input (CSRGraph.cpp:16-108): neighbours in edge-insertion order; the
    aggregation sums them in that order (SpMVNaiveFull semantics), which the
    oracle reproduces when given the CSR arrays."""
    el = sg.rmat(11, 8, seed=6)
    csr = sg.CSRGraph()
    csr.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    g_csr = csr.device_graph()
    g_csc = csc.device_graph()
    for tname in ("tree5", "spider7", "tree12"):
        n, edges = TEMPLATES[tname]
        P = O.Plan(n, edges)
        t = sg.Graph(n, edges)
        raw = sg.count(g_csr, t, 2, 70, exact=True)
        for i in range(2):
            colors = O.colors(70 + i, csr.getNumVertices(), n)
            r_o = O.count_coloring(csr.getIndexRow(), csr.getIndexCol(), P, colors)
            assert rel(raw[i], r_o) <= 1e-12, (tname, i, raw[i], r_o)
        # the same graph as CSC differs only in summation order
        raw_csc = sg.count(g_csc, t, 2, 70, exact=True)
        for a, b in zip(raw, raw_csc):
            assert rel(a, b) <= 1e-5, (tname, a, b)
    cm = sg.CountMat()
    cm.initialization(csr, None, 4, 2, 1, 0)
    cm.set_seed(70)
    assert cm.compute(sg.Graph(*TEMPLATES["tree5"])) > 0
