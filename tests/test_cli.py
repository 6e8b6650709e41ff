"""The sc-main drop-in CLI: the reference's argv and report lines."""
import os
import re
import subprocess

import numpy as np
import pytest

from tests.helpers import write_template

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "subgraph_b200", "bin", "sc-main")


def test_cli_usage_and_input_errors(tmp_path):
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    t = tmp_path / "t.fascia"
    write_template(str(t), 3, [(0, 1), (1, 2)])
    r = subprocess.run([CLI, str(tmp_path / "missing.txt"), str(t), "1", "1", "0", "0"], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 1 and "missing.txt" in r.stderr


def _report(stdout):
    vals = {}
    for key in ("Final raw count is", "Prob is", "Final count is"):
        m = re.search(re.escape(key) + r"\s+([0-9.eE+-]+)", stdout)
        vals[key] = float(m.group(1))
    assert re.search(r"Time for count per iter:\s+[0-9.]+ seconds", stdout)
    return vals


@pytest.mark.gpu
@pytest.mark.parametrize("binary", [False, True])
def test_cli_matches_reference_counts(tmp_path, golden, binary):
    c = next(c for c in golden.cases if c.template == "tree5" and c.graph == "rmat10")
    g = tmp_path / "g.txt"
    golden.write_graph("rmat10", str(g))
    t = tmp_path / "t.fascia"
    write_template(str(t), c.n, c.edges)
    env = dict(os.environ, SG_SEED_BASE=str(c.seed))
    graph_arg = str(g)
    if binary:   # write graph.data first, then load it (load_binary=1)
        r = subprocess.run([CLI, str(g), str(t), "1", "4", "0", "1"], capture_output=True, text=True, cwd=tmp_path,
                           env=env)
        assert r.returncode == 0, r.stderr
        graph_arg = str(tmp_path / "graph.data")
    r = subprocess.run([CLI, graph_arg, str(t), str(c.ncol), "4", "1" if binary else "0", "0", "1", "1"],
                       capture_output=True, text=True, cwd=tmp_path, env=env)
    assert r.returncode == 0, r.stderr
    got = _report(r.stdout)
    mean = float(np.mean(c.raw))
    assert abs(got["Final raw count is"] - mean) <= 1e-5 * mean
    assert abs(got["Prob is"] - 120 / 5 ** 5) < 1e-6
    expect = np.floor(mean / (120 / 5 ** 5) + 0.5)
    assert abs(got["Final count is"] - expect) <= 1e-5 * expect
