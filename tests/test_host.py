"""Host side of the product library (no GPU): loaders, CSC/CSR, graph.data,
DivideTemplates / IndexSys planning and the estimate, against the reference's
golden outputs and the oracle; malformed inputs come back as error codes."""
import random

import numpy as np
import pytest

import subgraph_b200 as sg
from oracle import oracle as O
from tests.helpers import TEMPLATES, prufer_tree, sha, write_graph, write_template


@pytest.mark.parametrize("gname", ["tiny", "holes", "rmat10", "rmat12"])
def test_edgelist_and_csc_match_reference(golden, gname, tmp_path):
    p = tmp_path / "g.txt"
    golden.write_graph(gname, str(p))
    el = sg.EdgeList(str(p))
    g = sg.CSCGraph()
    g.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    _, _, _, col, row = golden.graph(gname)
    assert np.array_equal(g.getIndexCol(), col)
    assert np.array_equal(g.getIndexRow(), row)
    assert np.array_equal(g.getDegList(), np.diff(col))


def test_hole_removal_shrinks_vertex_count(golden, tmp_path):
    p = tmp_path / "g.txt"
    golden.write_graph("holes", str(p))
    el = sg.EdgeList(str(p))
    case = next(c for c in golden.cases if c.graph == "holes")
    assert el.getNumVertices() == case.V == 7


def test_csr_build_keeps_insertion_order():
    src = np.array([0, 1, 2, 0, 3], np.int32)
    dst = np.array([1, 2, 0, 3, 3], np.int32)
    g = sg.CSRGraph()
    g.createFromEdgeListFile(4, 5, src, dst)
    # CSRGraph.cpp:82-96: row src gets dst, then row dst gets src, in edge order
    assert g.getIndexRow().tolist() == [0, 3, 5, 7, 10]
    assert g.getIndexCol().tolist() == [1, 2, 3, 0, 2, 1, 0, 0, 3, 3]


def test_graph_data_round_trip(golden, tmp_path):
    V, s, d, col, row = golden.graph("rmat10")
    g = sg.CSCGraph()
    g.createFromEdgeListFile(V, len(s), s, d)
    path = str(tmp_path / "graph.data")
    g.serialize(path)
    # layout of CSCGraph::serialize (CSCGraph.hpp:427-436)
    raw = np.fromfile(path, np.int32)
    nnz = len(row)
    assert raw[0] == len(s) and raw[1] == V
    assert np.array_equal(raw[2:2 + V], np.diff(col))
    assert np.array_equal(raw[2 + V:3 + 2 * V], col)
    assert np.array_equal(raw[3 + 2 * V:3 + 2 * V + nnz], row)
    assert np.all(np.fromfile(path, np.float32)[3 + 2 * V + nnz:] == 1.0)
    h = sg.CSCGraph()
    h.deserialize(path)
    assert np.array_equal(h.getIndexCol(), col) and np.array_equal(h.getIndexRow(), row)


def test_graph_data_truncated_is_an_error(golden, tmp_path):
    V, s, d, _, _ = golden.graph("tiny")
    g = sg.CSCGraph()
    g.createFromEdgeListFile(V, len(s), s, d)
    path = str(tmp_path / "graph.data")
    g.serialize(path)
    data = open(path, "rb").read()
    open(path, "wb").write(data[:-6])
    with pytest.raises(sg.SGError) as e:
        sg.CSCGraph().deserialize(path)
    assert e.value.code == 1


def test_truncated_edge_list_is_an_error(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("4\n3\n0 1\n1 2\n")
    with pytest.raises(sg.SGError) as e:
        sg.EdgeList(str(p))
    assert e.value.code == 1
    with pytest.raises(sg.SGError) as e:
        sg.EdgeList(str(tmp_path / "missing.txt"))
    assert e.value.code == 5


def test_edge_endpoint_out_of_range_is_an_error():
    with pytest.raises(sg.SGError):
        sg.CSCGraph().createFromEdgeListFile(3, 1, np.array([0], np.int32), np.array([5], np.int32))


@pytest.mark.parametrize("bad", [(3, [(0, 1)]), (3, [(0, 1), (0, 1)]), (1, []), (3, [(0, 1), (1, 5)]),
                                 (17, [(i, i + 1) for i in range(16)])])
def test_bad_templates_are_errors(bad):
    with pytest.raises(sg.SGError):
        sg.Graph(*bad)


def test_template_file_reader(tmp_path):
    p = tmp_path / "t.fascia"
    write_template(str(p), *TEMPLATES["tree12"])
    g = sg.Graph()
    g.read_enlist(str(p))
    assert g.get_vert_num() == 12 and g.edges == TEMPLATES["tree12"][1]


def test_plans_match_reference(golden):
    for c in golden.cases:
        g = sg.Graph(c.n, c.edges)
        dv = sg.DivideTemplates()
        dv.DivideTp(g)
        dv.sort_tps()
        ix = sg.IndexSys()
        ix.initialization(c.n, dv.get_subtps_num(), g, dv)
        assert dv.get_subtps_num() == len(c.subs)
        for s, ref in enumerate(c.subs):
            assert (dv.get_sub_size(s), dv.get_main_node_idx(s), dv.get_aux_node_idx(s), dv.get_parent(s)) == \
                (ref["size"], ref["main"], ref["aux"], ref["parent"]), (c.key, s)
            c2c, ms, as_ = ix.tables(s)
            if "c2c" in ref:
                assert c2c.tolist() == ref["c2c"]
                if ref["size"] > 1:
                    assert ms.tolist() == ref["msplit"] and as_.tolist() == ref["asplit"]
            else:
                assert sha(c2c) == ref["c2c_sha"]
                if ref["size"] > 1:
                    assert sha(ms) == ref["msplit_sha"] and sha(as_) == ref["asplit_sha"]
        if c.n <= 8:
            assert g.automorphisms() == c.aut


def test_plans_match_oracle_on_random_trees():
    """Breadth-first order + complement split rule == the reference's bubble sort and
    reversed-lex pairing, on 300 random trees with shuffled edge order."""
    rng = random.Random(11)
    for _ in range(300):
        n = rng.randint(2, 12)
        edges = prufer_tree(n, rng) if n > 2 else [(0, 1)]
        rng.shuffle(edges)
        edges = [(b, a) if rng.random() < 0.5 else (a, b) for a, b in edges]
        P = O.Plan(n, edges, automorphisms=n <= 8)
        g = sg.Graph(n, edges)
        dv = sg.DivideTemplates()
        dv.DivideTp(g)
        ix = sg.IndexSys()
        ix.initialization(n, 0, g, dv)
        assert dv.get_subtps_num() == P.nsub
        for s, si in enumerate(P.subs):
            assert (dv.get_sub_size(s), dv.get_main_node_idx(s), dv.get_aux_node_idx(s), dv.get_parent(s)) == \
                (si.size, si.main, si.aux, si.parent)
            c2c, ms, as_ = ix.tables(s)
            assert np.array_equal(c2c, si.c2c)
            if si.size > 1:
                assert np.array_equal(ms, si.msplit) and np.array_equal(as_, si.asplit)
        if n <= 8:
            assert g.automorphisms() == P.aut


def test_automorphisms_of_known_trees():
    assert sg.Graph(3, [(0, 1), (1, 2)]).automorphisms() == 2
    assert sg.Graph(5, [(0, 1), (0, 2), (0, 3), (0, 4)]).automorphisms() == 24
    assert sg.Graph(4, [(0, 1), (1, 2), (2, 3)]).automorphisms() == 2
    assert sg.Graph(7, TEMPLATES["spider7"][1]).automorphisms() == 6
    assert sg.Graph(12, TEMPLATES["tree12"][1]).automorphisms() == 2   # branches 6-7 and 10-11 at 5


def test_automorphisms_match_networkx_up_to_16():
    nx = pytest.importorskip("networkx")
    from networkx.algorithms.isomorphism import GraphMatcher
    rng = random.Random(3)
    for _ in range(60):
        n = rng.randint(3, 16)
        edges = prufer_tree(n, rng)
        G = nx.Graph(edges)
        expect = sum(1 for _ in GraphMatcher(G, G).isomorphisms_iter())
        assert sg.Graph(n, edges).automorphisms() == expect


def test_estimate_formula():
    raw = np.array([1.0e6, 1.2e6, 0.9e6])
    k = 5
    expect = np.floor(raw.mean() / (120 / 5 ** 5) + 0.5)
    assert sg.estimate(raw, k) == expect
    assert sg.estimate(raw, k, 2) == np.floor(raw.mean() / (2 * 120 / 5 ** 5) + 0.5)


def test_rmat_generator_shape():
    el = sg.rmat(12, 8, seed=1)
    V = el.getNumVertices()
    s, d = el.getSrcList(), el.getDstList()
    assert V == 4096
    assert np.all(s < d)                               # canonical, no self loops
    assert len(np.unique(s.astype(np.int64) * V + d)) == len(s)   # no duplicates
    assert max(s.max(), d.max()) == V - 1              # no hole removal on reload
    deg = np.bincount(np.concatenate([s, d]), minlength=V)
    assert deg.max() > 20 * deg.mean()                 # heavy tail
    el2 = sg.rmat(12, 8, seed=1)
    assert np.array_equal(el2.getSrcList(), s)        # seeded


def test_text_round_trip(tmp_path):
    el = sg.rmat(8, 4, seed=3)
    p = str(tmp_path / "g.txt")
    el.write(p)
    el2 = sg.EdgeList(p)
    assert el2.getNumVertices() == el.getNumVertices()
    assert np.array_equal(el2.getSrcList(), el.getSrcList())


def test_table_arena_slots_keep_32_byte_rows():
    """The aggregation reads gathered tables with 256-bit loads, so every table
    must start 32-byte aligned for any vertex count: the arena of every plan
    is a whole number of 8-unit slots (a unit is V elements)."""
    import ctypes
    from subgraph_b200._lib import lib
    rng = random.Random(29)
    trees = [TEMPLATES[t] for t in ("p3", "tree5", "spider7", "tree12")]
    trees += [(n, prufer_tree(n, rng)) for n in (rng.randint(3, 16) for _ in range(60))]
    for n, edges in trees:
        g = sg.Graph(n, edges)
        units = ctypes.c_int64()
        assert lib().sg_plan_info(g.plan, None, None, None, ctypes.byref(units)) == 0
        assert units.value > 0 and units.value % 8 == 0, (n, edges, units.value)


def test_csr_build_matches_reference():
    """CSRGraph::createFromEdgeListFile (CSRGraph.cpp:16-108): the library's CSR
    arrays equal the compiled reference's, including a graph whose edge file
    is unsorted with mixed orientation (neighbours in insertion order)."""
    from tests.helpers import GoldenFlags
    gf = GoldenFlags()
    for name in ("tiny", "rmat10s"):
        V, src, dst = gf.edges(name)
        row, col = gf.csr(name)
        g = sg.CSRGraph()
        g.createFromEdgeListFile(V, len(src), src, dst)
        assert np.array_equal(g.getIndexRow(), row), name
        assert np.array_equal(g.getIndexCol(), col), name


def _signature(P, s, scaled):
    """A sub's table signature: its rooted split structure and whether the
    1e-12-scaled sub lies below it (the oracle's own DivideTemplates)."""
    if P.subs[s].size == 1:
        return "1"
    return "(" + _signature(P, P.subs[s].main, scaled) + "," + _signature(P, P.subs[s].aux, scaled) + ")" + (
        "s" if s == scaled else "")


def test_shared_tables_are_subs_of_equal_signature():
    """A sub reuses the table of an earlier-processed sub exactly when both have
    the same split structure below them and the same relation to the scaled
    sub (the 12-vertex tree: its three unscaled 2-colour subs share one table;
    a 9-vertex tree whose size-3 subs differ only by the scaled sub beneath one
    of them shares nothing)."""
    t12 = sg.Graph(*TEMPLATES["tree12"])
    same = t12.shared_tables()
    assert [s for s, x in enumerate(same) if x >= 0] == [5, 11] and same[5] == same[11] == 16
    t9 = sg.Graph(9, [(2, 3), (4, 1), (7, 1), (1, 0), (0, 6), (6, 5), (5, 3), (3, 8)])
    assert all(x < 0 for x in t9.shared_tables())
    rng = random.Random(77)
    for _ in range(60):
        n = rng.randint(3, 14)
        edges = prufer_tree(n, rng)
        t = sg.Graph(n, edges)
        same = t.shared_tables()
        P = O.Plan(n, edges)
        order = [s for s in range(len(P.subs) - 1, -1, -1) if P.subs[s].size > 1]
        scaled = order[0]   # the first non-bottom sub processed (CountMat.cpp:813-822)
        seen = {}
        for s in order:
            if s == 0:
                assert same[s] == -1
                continue
            sig = _signature(P, s, scaled)
            if sig in seen:
                assert same[s] == seen[sig], (n, edges, s)
            else:
                assert same[s] == -1, (n, edges, s)
                seen[sig] = s
