"""The C++ drop-in headers (include/subgraph_b200/*.hpp): the reference's
class names and signatures (CountMat.hpp:32-35, CSCGraph.hpp:64-73,
CSRGraph.hpp:105-107, Graph.hpp:29, EdgeList.hpp:28-36) over the C ABI.

The sc-main CLI (subgraph_b200/csrc/sc_main.cpp) is written against these
headers with the reference main's own call sequence (sc-main.cpp:1620-1795),
so building it is the compile check; on the CPU its loading half runs
(graph.data written by the headers' serialize equals the library's
sg_graph_data_write bytes, and deserialize reads it back); on the GPU its
counts match the compiled reference for the CSC and the CSR branch.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import subgraph_b200 as sg
from tests.helpers import GoldenFlags, write_graph, write_template

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "subgraph_b200", "bin", "sc-main")
INC = os.path.join(ROOT, "include")


def _cxx():
    return shutil.which("g++") or "/usr/bin/g++"


def test_headers_compile_standalone(tmp_path):
    """Every drop-in header compiles on its own, and a translation unit using
    them the way the reference's main does (both graph types, both load paths)
    compiles and links against the library."""
    for h in sorted(os.listdir(os.path.join(INC, "subgraph_b200"))):
        src = tmp_path / f"only_{h}.cpp"
        src.write_text(f'#include "subgraph_b200/{h}"\nint main() {{ return 0; }}\n')
        r = subprocess.run([_cxx(), "-std=c++17", "-fsyntax-only", "-Wall", "-Werror", "-I" + INC, str(src)],
                           capture_output=True, text=True)
        assert r.returncode == 0, (h, r.stderr)
    src = tmp_path / "calls.cpp"
    src.write_text(r'''
#include <fcntl.h>
#include <unistd.h>
#include "subgraph_b200/CountMat.hpp"
#include "subgraph_b200/EdgeList.hpp"
int main(int argc, char** argv) {
    string graph_name = argv[1], template_name = argv[2];
    int comp_thds = 4, iterations = 2, isPruned = 1, useSPMM = 1, vtuneStart = -1;
    bool calculate_automorphism = false, useMKL = false, useRcm = false;
    CSRGraph* csrInputG = argc > 3 ? new CSRGraph() : nullptr;
    CSCGraph<int32_t, float>* cscInputG = argc > 3 ? nullptr : new CSCGraph<int32_t, float>();
    Graph input_template;
    double startTime = utility::timer();
    if (argc > 4) {
        int input_file = open(graph_name.c_str(), O_CREAT|O_RDWR, 0666);
        if (csrInputG != nullptr) csrInputG->deserialize(input_file, useMKL, useRcm);
        else { cscInputG->deserialize(input_file); cscInputG->splitCSC(4*comp_thds); }
        close(input_file);
    } else {
        EdgeList elist(graph_name);
        if (csrInputG != nullptr)
            csrInputG->createFromEdgeListFile(elist.getNumVertices(), elist.getNumEdges(), elist.getSrcList(), elist.getDstList(), useMKL, useRcm, false);
        else {
            cscInputG->createFromEdgeListFile(elist.getNumVertices(), elist.getNumEdges(), elist.getSrcList(), elist.getDstList(), false);
            cscInputG->splitCSC(4*comp_thds);
        }
    }
    ofstream output_file("graph.data", ios::binary);
    if (csrInputG != nullptr) csrInputG->serialize(output_file); else cscInputG->serialize(output_file);
    output_file.close();
    printf("Prepare Datasets using %f secs\n", (utility::timer() - startTime));
    input_template.read_enlist(template_name);
    CountMat executor;
    executor.initialization(csrInputG, cscInputG, comp_thds, iterations, isPruned, useSPMM, vtuneStart, calculate_automorphism);
    double r = executor.compute(input_template, false);
    if (csrInputG != nullptr) delete csrInputG;
    if (cscInputG != nullptr) delete cscInputG;
    return r >= 0 ? 0 : 1;
}
''')
    exe = tmp_path / "calls"
    r = subprocess.run([_cxx(), "-std=c++17", "-Wall", "-I" + INC, str(src), "-o", str(exe),
                        "-L" + os.path.join(ROOT, "subgraph_b200"), "-lsubgraph_b200",
                        "-Wl,-rpath," + os.path.join(ROOT, "subgraph_b200")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("csr", [False, True])
def test_cli_graph_data_round_trip(tmp_path, csr):
    """write_binary=1 through the headers' serialize gives the library's
    graph.data bytes; load_binary=1 reads them back (up to the counting, which
    needs a GPU)."""
    gf = GoldenFlags()
    V, src, dst = gf.edges("rmat10s")
    g = tmp_path / "g.txt"
    write_graph(str(g), V, src, dst)
    t = tmp_path / "t.fascia"
    write_template(str(t), 3, [(0, 1), (1, 2)])
    env = dict(os.environ, SG_USE_CSR="1" if csr else "0")
    subprocess.run([CLI, str(g), str(t), "1", "1", "0", "1"], capture_output=True, text=True, cwd=tmp_path, env=env)
    data = (tmp_path / "graph.data").read_bytes()
    h = sg.CSRGraph() if csr else sg.CSCGraph()
    h.createFromEdgeListFile(V, len(src), src, dst)
    off, nbr = (h.getIndexRow(), h.getIndexCol()) if csr else (h.getIndexCol(), h.getIndexRow())
    expect = tmp_path / "expect.data"
    sg.lib().sg_graph_data_write(str(expect).encode(), V, len(src), off.ctypes.data, nbr.ctypes.data,
                                 h.getDegList().ctypes.data)
    assert data == expect.read_bytes()
    if csr:
        row, col = gf.csr("rmat10s")
        assert np.array_equal(off, row) and np.array_equal(nbr, col)
    r = subprocess.run([CLI, str(tmp_path / "graph.data"), str(t), "1", "1", "1", "0"], capture_output=True,
                       text=True, cwd=tmp_path, env=env)
    assert f"{'CSR' if csr else 'CSC'} Format Total vertices is : {V}" in r.stdout


def _final_raw(stdout):
    m = re.search(r"Final raw count is\s+([0-9.eE+-]+|inf|nan)", stdout)
    return float(m.group(1))


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["spmv", "csr_spmv", "orig", "csr_orig"])
def test_cli_flag_variants_match_reference(tmp_path, variant):
    """The CLI's CSC branch and (SG_USE_CSR=1) its CSR branch with the
    reference's isPruned / useSPMM argv flags, against the compiled reference's
    raw counts: "Final raw count" is their mean (printed with %e)."""
    gf = GoldenFlags()
    c = next(c for c in gf.cases if c.variant == variant and c.template == "tree5" and c.graph != "tiny")
    V, src, dst = gf.edges(c.graph)
    g = tmp_path / "g.txt"
    write_graph(str(g), V, src, dst)
    t = tmp_path / "t.fascia"
    write_template(str(t), c.n, c.edges)
    env = dict(os.environ, SG_SEED_BASE=str(c.seed), SG_USE_CSR="1" if c.csr else "0")
    r = subprocess.run([CLI, str(g), str(t), str(c.ncol), "4", "0", "0", str(c.is_pruned), str(c.use_spmm)],
                       capture_output=True, text=True, cwd=tmp_path, env=env)
    assert r.returncode == 0, r.stderr
    got = _final_raw(r.stdout)
    mean = float(np.mean(c.raw))
    if not np.isfinite(mean):
        assert (np.isnan(got) and np.isnan(mean)) or got == mean
    else:
        assert abs(got - mean) <= 1e-5 * abs(mean), (got, mean)   # %e prints 7 significant digits
