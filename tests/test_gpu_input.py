"""Input preparation on the GPU: edge-list text parsed, the CSC of the
symmetrised adjacency built and an R-MAT graph generated on the device.  The
parsed and built graphs must equal the host loaders' arrays bit for bit
(EdgeList.cpp:34-116, CSCGraph.hpp:95-178) and count identically; the
generated graph must be a simple undirected R-MAT graph, the same for the
same seed."""
import numpy as np
import pytest

import subgraph_b200 as sg
from tests.helpers import TEMPLATES

pytestmark = pytest.mark.gpu


def _host_csc(V, src, dst):
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(V, len(src), np.asarray(src, np.int32), np.asarray(dst, np.int32))
    return csc


def _check_same(dg, csc):
    off, nbr = dg.csc()
    assert np.array_equal(off, csc.getIndexCol())
    assert np.array_equal(nbr, csc.getIndexRow())


def test_text_file_matches_host_loader(tmp_path):
    el = sg.rmat(12, 8, seed=3)
    p = tmp_path / "rmat12.txt"
    el.write(str(p))
    dg = sg.DeviceGraph.from_edge_list_file(str(p))
    host = sg.EdgeList(str(p))
    _check_same(dg, _host_csc(host.getNumVertices(), host.getSrcList(), host.getDstList()))
    # the same counts as the graph uploaded from host arrays
    g_host = sg.DeviceGraph(*(_host_csc(host.getNumVertices(), host.getSrcList(), host.getDstList()).getIndexCol(),
                              _host_csc(host.getNumVertices(), host.getSrcList(), host.getDstList()).getIndexRow()))
    for tname in ("tree5", "spider7"):
        t = sg.Graph(*TEMPLATES[tname])
        assert np.array_equal(sg.count(dg, t, 2, 9, exact=True), sg.count(g_host, t, 2, 9, exact=True))


def test_text_file_edge_cases(tmp_path):
    # holes (largest id != V-1), duplicate edges, a self loop, CRLF line ends,
    # extra blanks, a trailing line without newline and lines after E edges
    text = "10\r\n6\r\n3 7\r\n7  3\r\n5 5\r\n12 3\r\n 7 20\r\n3 12" + "\n99 98\n"
    p = tmp_path / "holes.txt"
    p.write_bytes(text.encode())
    dg = sg.DeviceGraph.from_edge_list_file(str(p))
    host = sg.EdgeList(str(p))
    assert dg.V == host.getNumVertices()
    _check_same(dg, _host_csc(host.getNumVertices(), host.getSrcList(), host.getDstList()))


def test_text_file_errors(tmp_path):
    cases = {"truncated.txt": "5\n3\n0 1\n1 2\n", "nospace.txt": "5\n2\n0 1\n12\n", "negative.txt": "5\n2\n0 1\n-1 2\n"}
    for name, text in cases.items():
        p = tmp_path / name
        p.write_text(text)
        with pytest.raises(sg.SGError):
            sg.DeviceGraph.from_edge_list_file(str(p))
    with pytest.raises(sg.SGError):
        sg.DeviceGraph.from_edge_list_file(str(tmp_path / "missing.txt"))


def test_edges_build_matches_host_and_rejects_bad_ids():
    el = sg.rmat(13, 6, seed=8)
    V, src, dst = el.getNumVertices(), el.getSrcList(), el.getDstList()
    # duplicates and self loops are kept in both builds
    src = np.concatenate([src, src[:50], np.array([4, 4], np.int32)])
    dst = np.concatenate([dst, dst[:50], np.array([4, 9], np.int32)])
    dg = sg.DeviceGraph.from_edges(V, src, dst)
    _check_same(dg, _host_csc(V, src, dst))
    with pytest.raises(sg.SGError):
        sg.DeviceGraph.from_edges(V, np.array([0, V], np.int32), np.array([1, 2], np.int32))


def test_rmat_on_device_is_simple_symmetric_and_seeded():
    g1 = sg.DeviceGraph.from_rmat(14, 8, seed=5)
    g2 = sg.DeviceGraph.from_rmat(14, 8, seed=5)
    g3 = sg.DeviceGraph.from_rmat(14, 8, seed=6)
    off, nbr = g1.csc()
    assert g1.V == 1 << 14
    assert np.array_equal(off, g2.csc()[0]) and np.array_equal(nbr, g2.csc()[1])
    assert not np.array_equal(nbr[: min(len(nbr), g3.nnz)], g3.csc()[1][: min(len(nbr), g3.nnz)])
    deg = np.diff(off)
    cols = np.repeat(np.arange(g1.V), deg)
    assert np.all(nbr != cols)                                    # no self loops
    key = cols.astype(np.int64) << 32 | nbr
    assert np.all(np.diff(key) > 0)                               # rows ascending, no duplicates
    rev = np.sort(nbr.astype(np.int64) << 32 | cols)
    assert np.array_equal(np.sort(key), rev)                      # symmetric
    assert deg[-1] > 0                                            # vertex V-1 in use
    assert 0.5 * 8 * g1.V < g1.nnz / 2 <= 8 * g1.V                # deduplicated draws
    # counts on it agree with the same arrays uploaded from the host
    gh = sg.DeviceGraph(off, nbr)
    t = sg.Graph(*TEMPLATES["tree5"])
    assert np.array_equal(sg.count(g1, t, 2, 3, exact=True), sg.count(gh, t, 2, 3, exact=True))


def test_out_of_range_neighbour_id_is_an_error():
    """Neighbour ids are range-checked on the device while the graph is
    relabelled: an id outside [0, V) fails the upload with the entry's index
    (the first bad one) and leaves the device usable."""
    off = np.array([0, 2, 3, 5, 6], np.int32)
    nbr = np.array([1, 3, 0, 0, 7, 2], np.int32)   # entry 4 names vertex 7 of 4
    with pytest.raises(sg.SGError, match="out of range at entry 4"):
        sg.DeviceGraph(off, nbr)
    nbr[4] = -1
    with pytest.raises(sg.SGError, match="out of range at entry 4"):
        sg.DeviceGraph(off, nbr)
    nbr[4] = 3
    g = sg.DeviceGraph(off, nbr)
    t = sg.Graph(*TEMPLATES["p3"])
    assert np.all(np.isfinite(sg.count(g, t, 2, 5)))
