"""sg_colors_noalloc, the coloring entry point for callers that cannot allocate
device memory (their memory comes from their own pool, or an allocation's
implicit synchronisation is not acceptable): it writes into a device buffer
the caller owns and keeps its scratch in a fixed array inside the library.

Checked through the C ABI against sg_colors on two calls in a row (different
sizes and seeds), so the second call cannot lean on the first one's output;
at the largest size the array admits (2^26 vertices, the last jump-table
entry included); and after the first call, that a call only enqueues its
kernel: it returns while the stream is still busy with earlier work.
This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import subgraph_b200 as sg
from subgraph_b200._lib import SG_ERR_INVALID, SG_OK, lib

pytestmark = pytest.mark.gpu


def _noalloc(V, k, seed, out, stream):
    return lib().sg_colors_noalloc(V, k, seed & 0xFFFFFFFF, ctypes.c_void_p(out.data_ptr()),
                                   ctypes.c_void_p(stream.cuda_stream))


def _expected(V, k, seed):
    g = sg.DeviceGraph(np.zeros(V + 1, np.int32), np.zeros(0, np.int32))
    out = g.colors(k, seed)
    del g
    return out


def test_noalloc_colors_match_sg_colors_on_two_calls():
    import torch
    stream = torch.cuda.Stream()
    for V, k, seed in ((70001, 12, 7), (3000, 5, 2**31 + 9)):
        expect = _expected(V, k, seed)
        out = torch.full((V,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert _noalloc(V, k, seed, out, stream) == SG_OK, lib().sg_last_error()
        stream.synchronize()
        assert np.array_equal(out.cpu().numpy(), expect), (V, k, seed)


def test_noalloc_at_the_largest_size():
    import torch
    V, k, seed = 1 << 26, 12, 11
    expect = _expected(V, k, seed)
    out = torch.full((V,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    assert _noalloc(V, k, seed, out, stream) == SG_OK, lib().sg_last_error()
    stream.synchronize()
    got = out.cpu().numpy()
    assert np.array_equal(got, expect)
    assert np.array_equal(got[-1024:], expect[-1024:])   # the last block's jump polynomial


def test_noalloc_later_calls_only_enqueue():
    import torch
    stream = torch.cuda.Stream()
    V, k = 50000, 7
    out = torch.zeros(V, dtype=torch.int32, device="cuda")
    assert _noalloc(V, k, 3, out, stream) == SG_OK, lib().sg_last_error()   # set-up (if not done yet)
    stream.synchronize()
    for seed in (4, 5):
        with torch.cuda.stream(stream):
            torch.cuda._sleep(200_000_000)          # keeps the stream busy for about 0.1 s
        assert _noalloc(V, k, seed, out, stream) == SG_OK, lib().sg_last_error()
        busy = not stream.query()
        stream.synchronize()
        assert busy, "the call waited for the stream"
        assert np.array_equal(out.cpu().numpy(), _expected(V, k, seed))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    out = torch.zeros(4, dtype=torch.int32, device="cuda")
    st = _noalloc((1 << 26) + 1, 3, 1, out, torch.cuda.current_stream())
    assert st == SG_ERR_INVALID
    assert b"2^26" in lib().sg_last_error()
