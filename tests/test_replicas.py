"""Replica (multi-GPU) host logic on CPU: world-size-2 gloo process group, each
rank counting its share of the colorings with the CPU oracle standing in for
its GPU; the gathered counts must equal a single-process run in order."""
import os
import socket

import numpy as np
import pytest

from subgraph_b200.replicas import count_replicas, shard


def test_shard_partitions_contiguously():
    for n in (0, 1, 5, 16, 17):
        for world in (1, 2, 3, 8):
            got = [shard(n, world, r) for r in range(world)]
            assert sum(c for _, c in got) == n
            pos = 0
            for first, c in got:
                assert first == pos
                pos += c
            assert max(c for _, c in got) - min(c for _, c in got) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, seed, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import oracle as O
    from tests.helpers import Golden, TEMPLATES
    gd = Golden()
    _, _, _, col, row = gd.graph("rmat10")
    nt, edges = TEMPLATES["tree5"]
    P = O.Plan(nt, edges)

    def count_fn(first_seed, cnt):
        return np.array([O.count_coloring(col, row, P, O.colors(first_seed + i, len(col) - 1, nt))
                         for i in range(cnt)])

    raw = count_replicas(count_fn, n, seed)
    np.save(os.path.join(out_dir, f"raw{rank}.npy"), raw)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("n", [5, 2])
def test_two_rank_gloo_gather_matches_single_process(tmp_path, golden, n):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, n, 7, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    c = next(c for c in golden.cases if c.template == "tree5" and c.graph == "rmat10")
    r0 = np.load(tmp_path / "raw0.npy")
    r1 = np.load(tmp_path / "raw1.npy")
    assert np.array_equal(r0, r1) and len(r0) == n
    # colorings 7, 8, 9 are the golden ones (the reference's own counts)
    k = min(n, c.ncol)
    assert np.array_equal(r0[:k], c.raw[:k])


def test_single_process_passthrough():
    calls = []

    def count_fn(seed, cnt):
        calls.append((seed, cnt))
        return np.arange(cnt, dtype=np.float64) + seed

    out = count_replicas(count_fn, 4, 10)
    assert calls == [(10, 4)] and out.tolist() == [10.0, 11.0, 12.0, 13.0]
