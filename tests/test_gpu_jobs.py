"""Job streams: one coloring each of jobs with different templates on one graph,
their stage launches spread over CUDA streams (default) or all their
sub-template stages in one persistent work queue.  Every job must give what
the plain form gives for its template and seed (exact mode: the reference's
arithmetic, 1e-12 for the FP64 sum order), in every count mode, with hub
chunking, and report a latency per job."""
import random

import numpy as np
import pytest

import subgraph_b200 as sg
from oracle import oracle as O
from tests.helpers import TEMPLATES, prufer_tree, rel

pytestmark = pytest.mark.gpu


def _csc(scale, ef, seed):
    el = sg.rmat(scale, ef, seed=seed)
    csc = sg.CSCGraph()
    csc.createFromEdgeListFile(el.getNumVertices(), el.getNumEdges(), el.getSrcList(), el.getDstList())
    return csc


def _jobs(rng, n):
    out = []
    for _ in range(n):
        k = rng.randint(3, 10)
        out.append((k, prufer_tree(k, rng)))
    return out


@pytest.mark.parametrize("persistent", [False, True])
def test_jobs_exact_match_oracle_and_plain(persistent):
    csc = _csc(11, 8, 3)
    g = csc.device_graph()
    rng = random.Random(5)
    jobs = _jobs(rng, 20) + [TEMPLATES["tree12"], TEMPLATES["spider7"], TEMPLATES["p3"]]
    tmpl = [sg.Graph(n, e) for n, e in jobs]
    seeds = [300 + 7 * j for j in range(len(jobs))]
    raw, lat = sg.count_jobs(g, tmpl, seeds, exact=True, return_latency=True, persistent=persistent)
    for j, ((n, e), t, s) in enumerate(zip(jobs, tmpl, seeds)):
        r_o = O.count_coloring(csc.getIndexCol(), csc.getIndexRow(), O.Plan(n, e), O.colors(s, csc.getNumVertices(), n))
        assert rel(raw[j], r_o) <= 1e-12, (j, n, e, raw[j], r_o)
        plain = sg.count(g, t, 1, s, exact=True)[0]
        assert rel(raw[j], plain) <= 1e-12, (j, raw[j], plain)
    assert np.all(lat > 0)


@pytest.mark.parametrize("persistent", [False, True])
def test_jobs_modes_and_hubs_match_plain(persistent):
    csc = _csc(13, 8, 4)
    g = csc.device_graph()
    rng = random.Random(9)
    jobs = _jobs(rng, 12) + [TEMPLATES["tree12"]]
    tmpl = [sg.Graph(n, e) for n, e in jobs]
    seeds = list(range(40, 40 + len(jobs)))
    for mode in (sg.MODE_REFERENCE, sg.MODE_FP64, sg.MODE_ORIGINAL_CSR):
        raw = sg.count_jobs(g, tmpl, seeds, mode=mode, exact=True, persistent=persistent)
        for j, (t, s) in enumerate(zip(tmpl, seeds)):
            assert rel(raw[j], sg.count(g, t, 1, s, mode=mode, exact=True)[0]) <= 1e-12, (mode, j)
    # fast path with hub chunks (vertices of degree > 32)
    raw, lat, st = sg.count_jobs(g, tmpl, seeds, hub_threshold=32, return_latency=True, return_stats=True,
                                 persistent=persistent)
    for j, (t, s) in enumerate(zip(tmpl, seeds)):
        assert rel(raw[j], sg.count(g, t, 1, s, hub_threshold=32)[0]) <= 1e-6, j
    assert np.all(lat > 0) and lat.max() <= st["device_ms"] * 1.01


def test_jobs_argument_errors():
    g = _csc(8, 4, 1).device_graph()
    t = sg.Graph(*TEMPLATES["p3"])
    with pytest.raises(ValueError):
        sg.count_jobs(g, [t, t], [1])
    with pytest.raises(sg.SGError):
        sg.count_jobs(g, [], [])


def test_job_streams_any_stream_count_matches_plain():
    """1, 3 and 8 streams (slots reused by later jobs of a stream), more jobs than streams."""
    csc = _csc(12, 8, 6)
    g = csc.device_graph()
    rng = random.Random(17)
    jobs = _jobs(rng, 19)
    tmpl = [sg.Graph(n, e) for n, e in jobs]
    seeds = [500 + j for j in range(len(jobs))]
    want = [sg.count(g, t, 1, s, exact=True)[0] for t, s in zip(tmpl, seeds)]
    for streams in (1, 3, 8):
        raw = sg.count_jobs(g, tmpl, seeds, exact=True, streams=streams)
        for j in range(len(jobs)):
            assert rel(raw[j], want[j]) <= 1e-12, (streams, j)
