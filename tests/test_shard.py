"""Batches over several ranks: partition balance, and the gather of every
rank's tetrahedra back into cloud order, with two gloo ranks on CPU (the GPU
triangulation is replaced by a deterministic stand-in per cloud)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from gstar4d_b200 import shard
from gstar4d_b200.api import TET_DTYPE


def fake_triangulate(points, offsets):
    """One 'tetrahedron' per 3 points of each cloud, filled from the cloud's
    first point so that every cloud's block is recognisable."""
    blocks, counts = [], []
    for c in range(len(offsets) - 1):
        p = points[offsets[c]:offsets[c + 1]]
        k = len(p) // 3
        b = np.zeros(k, TET_DTYPE)
        b["v"] = (p[0, 0] * 1e6).astype(np.int64) % 100000 + np.arange(k)[:, None]
        b["opp"] = np.arange(k)[:, None] - 1
        blocks.append(b)
        counts.append(k)
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return (np.concatenate(blocks) if blocks else np.zeros(0, TET_DTYPE)), offs


def _batch():
    rng = np.random.default_rng(3)
    sizes = rng.integers(5, 400, size=37)
    pts = rng.random((int(sizes.sum()), 3))
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    return pts, offs


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pts, offs = _batch()
        tets, toffs = shard.triangulate_batch_distributed(pts, offs, fake_triangulate, dst=0)
        if rank == 0:
            np.savez(out_path, tets=tets.view(np.int32).reshape(-1, 8), toffs=toffs)
        else:
            assert tets is None and toffs is None
    finally:
        dist.destroy_process_group()


def test_partition_balances_point_counts():
    sizes = np.random.default_rng(1).integers(64, 50000, size=4096)
    parts = shard.partition_clouds(sizes, 8)
    assert sorted(np.concatenate(parts).tolist()) == list(range(4096))
    loads = [sizes[p].sum() for p in parts]
    assert max(loads) - min(loads) <= sizes.max()


def test_two_rank_gather_restores_cloud_order(tmp_path):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "r0.npz")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    pts, offs = _batch()
    exp, eoffs = fake_triangulate(pts, offs)
    assert np.array_equal(got["toffs"], eoffs)
    assert np.array_equal(got["tets"], exp.view(np.int32).reshape(-1, 8))
