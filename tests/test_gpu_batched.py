"""The batched form: colorings of a batch run in one persistent launch over a
work queue (replayed from a CUDA graph).  It must give the plain form's
results, handle a final partial batch, and turn a dependency wait that never
completes into SG_ERR_TIMEOUT without losing the CUDA context."""
import numpy as np
import pytest

import subgraph_b200 as sg
from tests.helpers import TEMPLATES, rel

pytestmark = pytest.mark.gpu


def _graph(golden, name):
    _, _, _, col, row = golden.graph(name)
    return sg.DeviceGraph(col, row)


def test_batched_exact_matches_reference(golden):
    """Exact mode, 3 colorings in batches of 2 (a full and a partial batch)."""
    for tname in ("tree5", "spider7", "tree12", "p3"):
        c = next(c for c in golden.cases if c.template == tname and c.graph == "rmat10")
        g = _graph(golden, c.graph)
        t = sg.Graph(c.n, c.edges)
        raw = sg.count(g, t, c.ncol, c.seed, batch=2, exact=True)
        for i in range(c.ncol):
            assert rel(raw[i], c.raw[i]) <= 1e-12, (tname, i, raw[i], c.raw[i])


def test_batched_fast_close_to_plain(golden):
    c = next(c for c in golden.cases if c.template == "tree12" and c.graph == "rmat12")
    g = _graph(golden, c.graph)
    t = sg.Graph(c.n, c.edges)
    plain = sg.count(g, t, 5, 3)
    batched = sg.count(g, t, 5, 3, batch=4)
    again = sg.count(g, t, 5, 3, batch=4)          # replayed graph
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
    batched = sg.count(g, t, 4, 11, hub_threshold=32, batch=4)
    for a, b in zip(batched, plain):
        assert rel(a, b) <= 1e-6
    p64 = sg.count(g, t, 2, 11, mode=sg.MODE_FP64, exact=True)
    b64 = sg.count(g, t, 2, 11, mode=sg.MODE_FP64, exact=True, batch=2)
    assert np.array_equal(p64, b64)


def test_batched_wait_timeout_is_an_error_and_context_survives(golden):
    c = next(c for c in golden.cases if c.template == "tree5" and c.graph == "rmat10")
    g = _graph(golden, c.graph)
    t = sg.Graph(c.n, c.edges)
    with pytest.raises(sg.SGError) as e:
        sg.count(g, t, 2, c.seed, batch=2, wait_limit_ms=200, test_unsatisfiable_wait=True)
    assert e.value.code == 4
    raw = sg.count(g, t, c.ncol, c.seed, batch=2, exact=True)
    assert all(rel(a, b) <= 1e-12 for a, b in zip(raw, c.raw))
