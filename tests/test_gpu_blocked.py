"""The register-blocked eMA (outputs grouped by (|s|+1)-color supersets, the
held family in registers): every output receives its products in split
order, so its values must be bit-identical to the per-output split loop and
to the reference's arithmetic."""
import random

import numpy as np
import pytest

import subgraph_b200 as sg
from oracle import oracle as O
from tests.helpers import TEMPLATES, prufer_tree, rel

pytestmark = pytest.mark.gpu


def _graph(scale, ef, seed):
    el = sg.rmat(scale, ef, seed=seed)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    return csc


def test_blocked_equals_split_loop_and_reference(golden):
    for tname in ("tree12", "spider7", "tree5"):
        for c in [c for c in golden.cases if c.template == tname]:
            _, _, _, col, row = golden.graph(c.graph)
            g = sg.DeviceGraph(col, row)
            t = sg.Graph(c.n, c.edges)
            a = sg.count(g, t, c.ncol, c.seed, exact=True, autotune=False, blocked=True)
            b = sg.count(g, t, c.ncol, c.seed, exact=True, autotune=False, blocked=False)
            assert np.array_equal(a, b), (c.key, a, b)
            for i in range(c.ncol):
                assert rel(a[i], c.raw[i]) <= 1e-12, (c.key, i)


def test_blocked_random_trees_against_oracle():
    """Random Pruefer trees of 4..12 vertices: many (|s|, |main|) shapes."""
    csc = _graph(10, 8, 9)
    g = csc.device_graph()
    rng = random.Random(23)
    for i in range(16):
        n = rng.randint(4, 12)
        edges = prufer_tree(n, rng)
        t = sg.Graph(n, edges)
        a = sg.count(g, t, 1, 90 + i, exact=True, autotune=False, blocked=True)
        b = sg.count(g, t, 1, 90 + i, exact=True, autotune=False, blocked=False)
        assert np.array_equal(a, b), (n, edges)
        P = O.Plan(n, edges)
        r_o = O.count_coloring(csc.getIndexCol(), csc.getIndexRow(), P, O.colors(90 + i, csc.getNumVertices(), n))
        assert rel(a[0], r_o) <= 1e-12, (n, edges, a[0], r_o)


def test_blocked_in_tuned_fast_path():
    """The autotuner may pick blocked shapes; the fast path stays within 1e-6 of exact."""
    csc = _graph(13, 8, 4)
    g = csc.device_graph()
    t = sg.Graph(*TEMPLATES["tree12"])
    fast = sg.count(g, t, 2, 5)
    exact = sg.count(g, t, 2, 5, exact=True)
    for a, b in zip(fast, exact):
        assert rel(a, b) <= 1e-6


def test_rooted_form_equals_full_form(golden):
    """The rooted form of the register-blocked eMA (a vertex of color c computes
    only the sets and splits holding c, over the other k-1 colors) gives the
    full form's values in exact mode, with and without hub rows (table-level
    bit-exactness of the rooted form is covered by the golden table tests, whose
    parity helper takes the rooted form wherever a stage has one)."""
    rng = random.Random(5)
    trees = [TEMPLATES["tree12"], TEMPLATES["spider7"], TEMPLATES["tree5"]]
    trees += [(n, prufer_tree(n, rng)) for n in [rng.randint(5, 12) for _ in range(10)]]
    for gname in ("rmat10", "rmat12"):
        _, _, _, col, row = golden.graph(gname)
        g = sg.DeviceGraph(col, row)
        for n, edges in trees:
            t = sg.Graph(n, edges)
            for hub in (0, 16):
                a = sg.count(g, t, 2, 17, exact=True, hub_threshold=hub)
                b = sg.count(g, t, 2, 17, exact=True, hub_threshold=hub, rooted=False)
                # per-vertex values are identical; only the FP64 sum of tile
                # partials may differ in order if the two runs tile the root differently
                assert all(rel(x, y) <= 1e-12 for x, y in zip(a, b)), (gname, n, edges, hub, a, b)


def test_flat_aggregation_equals_grouped(golden):
    """The flat aggregation (the tile's (vertex, chunk group) items spread over
    all threads, each vertex walking only the column chunks that hold a set
    lacking its color) gives the grouped form's values bit for bit: untuned
    shapes (flat by default where it applies), FP32 exact and fast paths and
    FP64 tables, with and without hub rows; exact FP32 also against the
    reference's raw counts."""
    rng = random.Random(41)
    trees = [TEMPLATES["tree12"], TEMPLATES["spider7"], TEMPLATES["tree5"]]
    trees += [(n, prufer_tree(n, rng)) for n in [rng.randint(5, 12) for _ in range(6)]]
    for gname in ("rmat10", "rmat12"):
        _, _, _, col, row = golden.graph(gname)
        g = sg.DeviceGraph(col, row)
        for n, edges in trees:
            t = sg.Graph(n, edges)
            for hub in (0, 16):
                for kw in (dict(exact=True), dict(exact=False), dict(mode=sg.MODE_FP64)):
                    a = sg.count(g, t, 2, 31, autotune=False, hub_threshold=hub, **kw)
                    b = sg.count(g, t, 2, 31, autotune=False, hub_threshold=hub, flat=False, **kw)
                    assert np.array_equal(a, b), (gname, n, edges, hub, kw, a, b)
    for c in [c for c in golden.cases if c.template in ("tree12", "spider7")]:
        _, _, _, col, row = golden.graph(c.graph)
        g = sg.DeviceGraph(col, row)
        a = sg.count(g, sg.Graph(c.n, c.edges), c.ncol, c.seed, exact=True, autotune=False)
        for i in range(c.ncol):
            assert rel(a[i], c.raw[i]) <= 1e-12, (c.key, i)
