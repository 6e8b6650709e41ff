"""The CountMat flag variants and the CSR input path on the sm_100a kernels,
against the compiled reference's own results (tests/golden/golden_flags.*):

  spmv      isPruned=1 useSPMM=0, CSC graph  -> SG_MODE_REFERENCE
  orig      isPruned=0, CSC graph            -> SG_MODE_ORIGINAL (the SpMV
            buffer accumulates over splits, sub-templates and colorings,
            CountMat.cpp:931; the results reach inf and NaN and must too)
  csr_spmv  isPruned=1 useSPMM=0, CSRGraph   -> SG_MODE_REFERENCE on the CSR
  csr_orig  isPruned=0, CSRGraph             -> SG_MODE_ORIGINAL_CSR

Exact mode (every neighbour list summed in order, products rounded then added):
every sub-template table of coloring 0 bit-identical to the reference's (NaNs
canonicalised), raw counts equal up to the order of the final FP64 sum
(relative 1e-12; inf and NaN exactly where the reference has them).  Also
through the CountMat mirror, whose isPruned=0 state carries from one
compute() to the next as the reference's _bufVec does.
"""
import numpy as np
import pytest

import subgraph_b200 as sg
from oracle import oracle as O
from tests.helpers import GoldenFlags, same_raw, sha_nan

pytestmark = pytest.mark.gpu

MODES = {"spmv": sg.MODE_REFERENCE, "orig": sg.MODE_ORIGINAL, "csr_spmv": sg.MODE_REFERENCE,
         "csr_orig": sg.MODE_ORIGINAL_CSR}


@pytest.fixture(scope="module")
def gf():
    return GoldenFlags()


_host = {}


def host_graph(gf, name, csr):
    key = (name, csr)
    if key not in _host:
        V, src, dst = gf.edges(name)
        h = sg.CSRGraph() if csr else sg.CSCGraph()
        h.createFromEdgeListFile(V, len(src), src, dst)
        _host[key] = h
    return _host[key]


def test_flag_variants_raw_counts(gf):
    for c in gf.cases:
        g = host_graph(gf, c.graph, c.csr).device_graph()
        t = sg.Graph(c.n, c.edges)
        raw = sg.count(g, t, c.ncol, c.seed, mode=MODES[c.variant], exact=True, hub_threshold=0)
        for i in range(c.ncol):
            assert same_raw(raw[i], c.raw[i], 1e-12), (c.variant, c.graph, c.template, i, raw[i], c.raw[i])


def test_flag_variants_tables_bit_exact(gf):
    n = 0
    for c in gf.cases:
        g = host_graph(gf, c.graph, c.csr).device_graph()
        t = sg.Graph(c.n, c.edges)
        for s, digest in c.table_sha.items():
            T = sg.debug_sub_table(g, t, c.seed, s, mode=MODES[c.variant], hub_threshold=0)
            assert sha_nan(T) == digest, (c.variant, c.graph, c.template, s)
            n += 1
    assert n > 40


def test_flag_variants_through_countmat(gf):
    """sg.CountMat with the reference's initialization flags and graph types."""
    for c in gf.cases:
        h = host_graph(gf, c.graph, c.csr)
        cm = sg.CountMat()
        cm.initialization(h if c.csr else None, None if c.csr else h, 4, c.ncol, c.is_pruned, c.use_spmm)
        cm.set_seed(c.seed)
        cm.compute(sg.Graph(c.n, c.edges))
        raw = cm.raw_counts()
        for i in range(c.ncol):
            assert same_raw(raw[i], c.raw[i], 1e-12), (c.variant, c.graph, c.template, i, raw[i], c.raw[i])


def test_original_state_carries_across_computes(gf):
    """isPruned=0 on a CSC graph: a second compute() on the same CountMat starts
    from the buffer the first one left (the reference never clears _bufVec),
    checked against the oracle running the same colorings back to back."""
    V, src, dst = gf.edges("rmat10")
    h = host_graph(gf, "rmat10", False)
    for tname, n, edges in (("p3", 3, [(0, 1), (1, 2)]), ("tree5", 5, [(0, 1), (1, 2), (2, 3), (1, 4)])):
        cm = sg.CountMat()
        cm.initialization(None, h, 4, 2, 0, 1)
        cm.set_seed(21)
        t = sg.Graph(n, edges)
        cm.compute(t)
        first = cm.raw_counts()
        cm.compute(t)
        second = cm.raw_counts()
        P = O.Plan(n, edges)
        col, row, _ = O.csc_build(V, src, dst)
        colors = [O.colors(21 + i, V, n) for i in range(2)]
        ref = O.count_colorings(col, row, P, colors + colors, O.MODE_ORIGINAL)
        for i in range(2):
            assert same_raw(first[i], ref[i], 1e-12), (tname, i)
            assert same_raw(second[i], ref[2 + i], 1e-12), (tname, i)
        # a fresh sg_count call starts from zeros (a fresh CountMat)
        raw = sg.count(h.device_graph(), t, 2, 21, mode=sg.MODE_ORIGINAL)
        assert all(same_raw(a, b, 1e-12) for a, b in zip(raw, ref[:2]))


def test_original_mode_ignores_batching(gf):
    """Mode 2 carries state from coloring to coloring, so a batched request runs
    its colorings in order and gives the plain form's results."""
    c = next(c for c in gf.cases if c.variant == "orig" and c.graph == "rmat10" and c.template == "tree5")
    g = host_graph(gf, c.graph, False).device_graph()
    t = sg.Graph(c.n, c.edges)
    for kw in (dict(batch=3), dict(batch=3, persistent=True)):
        raw = sg.count(g, t, c.ncol, c.seed, mode=sg.MODE_ORIGINAL, **kw)
        for i in range(c.ncol):
            assert same_raw(raw[i], c.raw[i], 1e-12), (kw, i)


def test_original_mode_rejected_in_job_streams(gf):
    g = host_graph(gf, "rmat10", False).device_graph()
    t = sg.Graph(3, [(0, 1), (1, 2)])
    with pytest.raises(sg.SGError) as e:
        sg.count_jobs(g, [t, t], [1, 2], mode=sg.MODE_ORIGINAL)
    assert e.value.code == 6
