"""The batched forms.

Persistent: the colorings of a batch run in one persistent launch over a
work queue (replayed from a CUDA graph).  Interleaved groups: the colorings
of a batch share table rows ([V][B][pitch]) and every stage launch serves
several of them.  Both must give the plain form's results, handle a final
partial batch; the persistent queue must turn a dependency wait that never
completes into SG_ERR_TIMEOUT without losing the CUDA context."""
import random

import numpy as np
import pytest

import subgraph_b200 as sg
from oracle import oracle as O
from tests.helpers import TEMPLATES, prufer_tree, rel

pytestmark = pytest.mark.gpu


def _rmat_graph(scale, ef, seed):
    el = sg.rmat(scale, ef, seed=seed)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    return csc


def _graph(golden, name):
    _, _, _, col, row = golden.graph(name)
    return sg.DeviceGraph(col, row)


def test_batched_exact_matches_reference(golden):
    """Exact mode, 3 colorings in batches of 2 (a full and a partial batch)."""
    for tname in ("tree5", "spider7", "tree12", "p3"):
        c = next(c for c in golden.cases if c.template == tname and c.graph == "rmat10")
        g = _graph(golden, c.graph)
        t = sg.Graph(c.n, c.edges)
        raw = sg.count(g, t, c.ncol, c.seed, batch=2, exact=True, persistent=True)
        for i in range(c.ncol):
            assert rel(raw[i], c.raw[i]) <= 1e-12, (tname, i, raw[i], c.raw[i])


def test_batched_fast_close_to_plain(golden):
    c = next(c for c in golden.cases if c.template == "tree12" and c.graph == "rmat12")
    g = _graph(golden, c.graph)
    t = sg.Graph(c.n, c.edges)
    plain = sg.count(g, t, 5, 3)
    batched = sg.count(g, t, 5, 3, batch=4, persistent=True)
    again = sg.count(g, t, 5, 3, batch=4, persistent=True)          # replayed graph
    assert np.array_equal(batched, again)
    for a, b in zip(batched, plain):
        assert rel(a, b) <= 1e-6


def test_batched_with_hubs_and_fp64():
    el = sg.rmat(13, 8, seed=4)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    g = csc.device_graph()
    t = sg.Graph(*TEMPLATES["spider7"])
    plain = sg.count(g, t, 4, 11, hub_threshold=32)
    batched = sg.count(g, t, 4, 11, hub_threshold=32, batch=4, persistent=True)
    for a, b in zip(batched, plain):
        assert rel(a, b) <= 1e-6
    p64 = sg.count(g, t, 2, 11, mode=sg.MODE_FP64, exact=True)
    b64 = sg.count(g, t, 2, 11, mode=sg.MODE_FP64, exact=True, batch=2, persistent=True)
    assert np.array_equal(p64, b64)


def test_batched_wait_timeout_is_an_error_and_context_survives(golden):
    c = next(c for c in golden.cases if c.template == "tree5" and c.graph == "rmat10")
    g = _graph(golden, c.graph)
    t = sg.Graph(c.n, c.edges)
    with pytest.raises(sg.SGError) as e:
        sg.debug_count_unsatisfiable_wait(g, t, 2, c.seed, batch=2, wait_limit_ms=200)
    assert e.value.code == 4
    raw = sg.count(g, t, c.ncol, c.seed, batch=2, exact=True, persistent=True)
    assert all(rel(a, b) <= 1e-12 for a, b in zip(raw, c.raw))


# ---------------------------------------------------------------------------
# interleaved groups
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("batch", [2, 3, 4, 16])
def test_grouped_exact_matches_reference(golden, batch):
    """Exact mode: every coloring of a group equals the reference's count (1e-12;
    only the FP64 sum of tile partials may differ in order)."""
    for tname in ("p3", "tree5", "spider7", "tree12"):
        for c in [c for c in golden.cases if c.template == tname and c.graph in ("rmat10", "rmat12")]:
            _, _, _, col, row = golden.graph(c.graph)
            g = sg.DeviceGraph(col, row)
            t = sg.Graph(c.n, c.edges)
            raw = sg.count(g, t, c.ncol, c.seed, batch=batch, exact=True)
            for i in range(c.ncol):
                assert rel(raw[i], c.raw[i]) <= 1e-12, (c.key, batch, i, raw[i], c.raw[i])


def test_grouped_matches_plain_with_hubs_and_modes():
    el = sg.rmat(13, 8, seed=4)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    g = csc.device_graph()
    for tname in ("spider7", "tree5", "tree12"):
        t = sg.Graph(*TEMPLATES[tname])
        for mode in (sg.MODE_REFERENCE, sg.MODE_FP64, sg.MODE_ORIGINAL_CSR):
            n = 2 if tname == "tree12" else 9
            plain = sg.count(g, t, n, 21, mode=mode, hub_threshold=32, exact=True)
            grouped = sg.count(g, t, n, 21, mode=mode, hub_threshold=32, exact=True, batch=4)
            for a, b in zip(grouped, plain):
                assert rel(a, b) <= 1e-12, (tname, mode, a, b)
        fast = sg.count(g, t, 5, 3, hub_threshold=32, batch=5)
        ref = sg.count(g, t, 5, 3, hub_threshold=32)
        for a, b in zip(fast, ref):
            assert rel(a, b) <= 1e-6, (tname, a, b)


def test_grouped_random_trees_against_oracle():
    csc = _rmat_graph(10, 8, 9)
    g = csc.device_graph()
    rng = random.Random(31)
    for i in range(8):
        n = rng.randint(3, 10)
        edges = prufer_tree(n, rng)
        P = O.Plan(n, edges)
        raw = sg.count(g, sg.Graph(n, edges), 3, 200 + 3 * i, exact=True, batch=3)
        for j in range(3):
            r_o = O.count_coloring(csc.getIndexCol(), csc.getIndexRow(), P,
                                   O.colors(200 + 3 * i + j, csc.getNumVertices(), n))
            assert rel(raw[j], r_o) <= 1e-12, (n, edges, j)


def test_grouped_large_group_matches_plain():
    """64 colorings in one group: colour histograms of more than 16 colorings per launch."""
    csc = _rmat_graph(12, 8, 13)
    g = csc.device_graph()
    for tname in ("spider7", "p3"):
        t = sg.Graph(*TEMPLATES[tname])
        plain = sg.count(g, t, 64, 40, exact=True)
        grouped = sg.count(g, t, 64, 40, exact=True, batch=64)
        for i, (a, b) in enumerate(zip(grouped, plain)):
            assert rel(a, b) <= 1e-12, (tname, i, a, b)
