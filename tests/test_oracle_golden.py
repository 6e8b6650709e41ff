"""Pins the CPU oracle (oracle/sg_oracle.c) to the compiled reference's outputs.

Every golden case was produced by the reference's own CountMat / CSCGraph /
EdgeList / DivideTemplates / IndexSys objects (tests/golden/make_golden.py).
The oracle must reproduce all of it exactly: colors, CSC arrays, the sub list
and index tables, every sub-template table of coloring 0 and the raw counts.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import sha


def _edgelist(golden, name, tmp_path):
    """The edge list as the reference's EdgeList reads it (hole removal)."""
    import subgraph_b200 as sg
    p = tmp_path / f"{name}.txt"
    golden.write_graph(name, str(p))
    el = sg.EdgeList(str(p))
    return el.getNumVertices(), el.getSrcList(), el.getDstList()


def test_glibc_stream_matches_host_libc():
    import ctypes
    libc = ctypes.CDLL("libc.so.6")
    for seed in (0, 1, 7, 2**31 + 3):
        libc.srand(ctypes.c_uint(seed))
        ref = np.array([libc.rand() for _ in range(2000)], np.int32)
        assert (O.glibc_rand(seed, 2000) == ref).all()


@pytest.mark.parametrize("gname", ["tiny", "holes", "rmat10", "rmat12"])
def test_oracle_csc_matches_reference(golden, gname, tmp_path):
    V, s, d = _edgelist(golden, gname, tmp_path)
    col, row, _ = O.csc_build(V, s, d)
    _, _, _, rcol, rrow = golden.graph(gname)
    assert np.array_equal(col, rcol) and np.array_equal(row, rrow)


def test_oracle_plans_match_reference(golden):
    for c in golden.cases:
        P = O.Plan(c.n, c.edges, automorphisms=c.n <= 8)
        assert P.nsub == len(c.subs), c.key
        for s, (mine, ref) in enumerate(zip(P.subs, c.subs)):
            assert (mine.size, mine.main, mine.aux, mine.parent, mine.L, mine.S) == \
                (ref["size"], ref["main"], ref["aux"], ref["parent"], ref["L"], ref["S"]), (c.key, s)
            if "c2c" in ref:
                assert mine.c2c.tolist() == ref["c2c"]
                if mine.size > 1:
                    assert mine.msplit.tolist() == ref["msplit"]
                    assert mine.asplit.tolist() == ref["asplit"]
            else:
                assert sha(mine.c2c.astype(np.int32)) == ref["c2c_sha"]
                if mine.size > 1:
                    assert sha(mine.msplit.astype(np.int32)) == ref["msplit_sha"]
                    assert sha(mine.asplit.astype(np.int32)) == ref["asplit_sha"]
        if c.n <= 8:
            assert P.aut == c.aut, c.key


def test_oracle_colors_and_counts_match_reference(golden, tmp_path):
    csc = {}
    for c in golden.cases:
        if c.graph not in csc:
            _, _, _, col, row = golden.graph(c.graph)
            csc[c.graph] = (col, row)
        col, row = csc[c.graph]
        P = O.Plan(c.n, c.edges)
        for i in range(c.ncol):
            colors = O.colors(c.seed + i, c.V, c.n)
            assert np.array_equal(colors, c.colors[i]), (c.key, i)
            raw = O.count_coloring(col, row, P, colors)
            # the same operations in the same order: equal to the last bit
            assert raw == c.raw[i], (c.key, i, raw, c.raw[i])


def test_oracle_tables_match_reference(golden):
    n_checked = 0
    for c in golden.cases:
        if not c.table_sha:
            continue
        _, _, _, col, row = golden.graph(c.graph)
        P = O.Plan(c.n, c.edges)
        colors = O.colors(c.seed, c.V, c.n)
        for s, digest in c.table_sha.items():
            T = O.sub_table(col, row, P, colors, s)
            assert sha(T) == digest, (c.key, s)
            n_checked += 1
    assert n_checked > 30


def test_oracle_estimate_matches_reference_formula(golden):
    c = next(c for c in golden.cases if c.template == "tree5" and c.graph == "rmat10")
    est = O.estimate(c.raw, c.n, 1)
    mean = float(np.mean(c.raw))
    assert est == np.floor(mean / (120.0 / 5 ** 5) + 0.5)


def test_oracle_fp64_mode_close_to_fp32(golden):
    """The FP64-table mode agrees with the reference's FP32 arithmetic to ~1e-6 on small graphs."""
    c = next(c for c in golden.cases if c.template == "tree12" and c.graph == "rmat10")
    _, _, _, col, row = golden.graph(c.graph)
    P = O.Plan(c.n, c.edges)
    colors = O.colors(c.seed, c.V, c.n)
    r64 = O.count_coloring(col, row, P, colors, mode=O.MODE_FP64)
    assert abs(r64 - c.raw[0]) / r64 < 1e-5


def test_planted_mistake_is_caught(golden):
    """A mistake planted in the oracle's input (one vertex recolored) moves the count off
    the reference value, so the exact comparisons above are able to fail."""
    c = next(c for c in golden.cases if c.template == "tree5" and c.graph == "rmat10")
    _, _, _, col, row = golden.graph(c.graph)
    P = O.Plan(c.n, c.edges)
    colors = O.colors(c.seed, c.V, c.n)
    hub = int(np.argmax(np.diff(col)))
    colors[hub] = (colors[hub] + 1) % c.n
    assert O.count_coloring(col, row, P, colors) != c.raw[0]


# ---------------------------------------------------------------------------
# CountMat flag variants and the CSR input path (golden_flags: the compiled
# reference with isPruned / useSPMM / CSRGraph)
# ---------------------------------------------------------------------------
def test_oracle_flag_variants_match_reference():
    from tests.helpers import GoldenFlags, same_raw
    gf = GoldenFlags()
    modes = {"spmv": O.MODE_REF, "orig": O.MODE_ORIGINAL, "csr_spmv": O.MODE_REF, "csr_orig": O.MODE_ORIGINAL_CSR}
    for c in gf.cases:
        V, src, dst = gf.edges(c.graph)
        if c.csr:
            off, nbr = gf.csr(c.graph)
        else:
            off, nbr, _ = O.csc_build(V, src, dst)
        assert np.array_equal(c.colors[0], O.colors(c.seed, c.V, c.n))
        P = O.Plan(c.n, c.edges)
        raw = O.count_colorings(off, nbr, P, [c.colors[i] for i in range(c.ncol)], modes[c.variant])
        for i in range(c.ncol):
            assert same_raw(raw[i], c.raw[i]), (c.variant, c.graph, c.template, i, raw[i], c.raw[i])


def test_useSPMM_flag_does_not_change_results(golden):
    """countNonBottomePruned (useSPMM=0) equals countNonBottomePrunedSPMM bit for
    bit in the reference: same graph, template and seeds in both fixture sets."""
    from tests.helpers import GoldenFlags
    gf = GoldenFlags()
    n = 0
    for c in gf.cases:
        if c.variant != "spmv":
            continue
        for g in golden.cases:
            if g.graph == c.graph and g.template == c.template and g.seed == c.seed:
                m = min(g.ncol, c.ncol)
                assert np.array_equal(g.raw[:m], c.raw[:m]), (c.graph, c.template)
                n += 1
    assert n >= 3
