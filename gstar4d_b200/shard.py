"""Batches over several GPUs: one process per GPU (torch.distributed), clouds
partitioned across ranks, no collective on the data path.

Clouds are independent, so each rank triangulates its share with the batched
entry point on its own GPU; the only exchange is the final gather of every
rank's tetrahedra to the destination rank (NCCL over NVLink on GPU ranks, gloo
on CPU ranks). Single clouds do not shard: across GPUs they run as replicas.
"""
import heapq

import numpy as np


def partition_clouds(sizes, world, cost=None):
    """Greedy longest-processing-time balance: clouds in decreasing cost go to
    the least-loaded rank. cost defaults to the point count (triangulation
    work grows about linearly with it). Returns one sorted index array per rank."""
    sizes = np.asarray(sizes, dtype=np.int64)
    c = np.asarray(cost if cost is not None else sizes, dtype=np.float64)
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in np.argsort(-c, kind="stable"):
        load, r = heapq.heappop(heap)
        parts[r].append(int(i))
        heapq.heappush(heap, (load + float(c[i]), r))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def _subset(points, offsets, idx):
    offs = np.zeros(len(idx) + 1, dtype=np.int64)
    chunks = []
    for k, c in enumerate(idx):
        a, b = int(offsets[c]), int(offsets[c + 1])
        chunks.append(points[a:b])
        offs[k + 1] = offs[k] + (b - a)
    pts = np.concatenate(chunks) if chunks else np.zeros((0, 3), np.float64)
    return np.ascontiguousarray(pts), offs


def triangulate_batch_distributed(points, offsets, triangulate, dst=0, group=None):
    """Every rank passes the whole batch (points, offsets); rank r triangulates
    the clouds partition_clouds assigns it with triangulate(points, offsets) ->
    (tets, tet_offsets) and the destination rank receives all tetrahedra in the
    original cloud order: (tets, tet_offsets) there, (None, None) elsewhere."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    sizes = np.diff(np.asarray(offsets, dtype=np.int64))
    parts = partition_clouds(sizes, world)
    mine = parts[rank]
    if len(mine):
        sub, sub_offs = _subset(points, offsets, mine)
        tets, toffs = triangulate(sub, sub_offs)
        counts = np.diff(np.asarray(toffs, dtype=np.int64))
        flat = np.ascontiguousarray(tets).view(np.int32).reshape(-1, 8) if len(tets) else np.zeros((0, 8), np.int32)
    else:
        counts = np.zeros(0, np.int64)
        flat = np.zeros((0, 8), np.int32)
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    # sizes first (every rank takes the same collective steps), then the payloads
    n_local = torch.tensor([len(flat)], dtype=torch.int64, device=device)
    n_all = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(n_all, n_local, group=group)
    n_all = [int(t.item()) for t in n_all]
    cap = max(max(n_all), 1)
    send = torch.zeros((cap, 8), dtype=torch.int32, device=device)
    if len(flat):
        send[: len(flat)] = torch.from_numpy(flat).to(device)
    recv = [torch.zeros((cap, 8), dtype=torch.int32, device=device) for _ in range(world)] if rank == dst else None
    dist.gather(send, recv, dst=dst, group=group)
    c_local = torch.zeros(max(len(p) for p in parts) or 1, dtype=torch.int64, device=device)
    c_local[: len(counts)] = torch.from_numpy(counts).to(device)
    c_recv = [torch.zeros_like(c_local) for _ in range(world)] if rank == dst else None
    dist.gather(c_local, c_recv, dst=dst, group=group)
    if rank != dst:
        return None, None
    from .api import TET_DTYPE
    per_cloud = [None] * len(sizes)
    for r in range(world):
        block = recv[r][: n_all[r]].cpu().numpy()
        cnt = c_recv[r][: len(parts[r])].cpu().numpy()
        o = np.concatenate([[0], np.cumsum(cnt)])
        for k, c in enumerate(parts[r]):
            per_cloud[c] = block[o[k]:o[k + 1]]
    out_offs = np.zeros(len(sizes) + 1, dtype=np.int64)
    out_offs[1:] = np.cumsum([len(b) for b in per_cloud])
    flat_all = np.concatenate(per_cloud) if len(per_cloud) else np.zeros((0, 8), np.int32)
    tets = np.ascontiguousarray(flat_all.astype(np.int32)).view(TET_DTYPE).reshape(-1)
    return tets, out_offs
