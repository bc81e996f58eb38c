"""The push rule of the voxel-block workset pairs, restated and checked on the CPU.

gstar4d_b200/csrc/g4d_block.cu: every point s of a voxel with several points
selects the block points whose squared distance (a float, the same from both
sides) is at most its threshold t(s), the K-th smallest of its block's
distances (all of them when there are fewer), minus the pairs already in its
workset; points that select nothing have t = -1. k_block_push then pushes the
pair (s, v) into both worksets from s when v is in s's selection and either
v > s or d(s, v) > t(v), and otherwise leaves it to v. Splaying needs the
worksets symmetric (each push goes into both worksets) and a pair pushed
twice wastes workset room, so no pair may be pushed twice; when no cap binds,
every pair of the union of the selections is pushed. (Where one side never
gathered the other, beyond the caps of 16 points per voxel and 128 block
points, the pair can be left out; splaying then inserts it.) The restatement
here follows the kernels' rule on random clouds, with the same caps and
nearer-voxels-first order, and stand-ins for the existing worksets
(symmetric, as they are).
"""
import random

import numpy as np

ORDER = sorted(((dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)),
               key=lambda o: abs(o[0]) + abs(o[1]) + abs(o[2]))


def _selections(P, vox, K, bucket):
    n = len(P)
    cells = {}
    for i, v in enumerate(map(tuple, vox)):
        cells.setdefault(v, []).append(i)
    thr = np.full(n, -1.0, np.float32)
    sel = [[] for _ in range(n)]
    for s in range(n):
        own = cells[tuple(vox[s])]
        if len(own) < 2:
            continue  # alone in its voxel: selects nothing
        block = []
        for o in ORDER:
            block.extend(cells.get(tuple(vox[s] + np.array(o)), [])[:16])
        block = block[:128]
        cand = [v for v in block if v != s]
        if not cand:
            continue
        d = np.array([np.float32(((P[s] - P[v]) ** 2).sum()) for v in cand], np.float32)
        t = np.float32(np.inf) if len(cand) <= K else np.sort(d)[K - 1]
        thr[s] = t
        sel[s] = [v for v, dv in zip(cand, d) if dv <= t and v not in bucket[s]]
    return thr, sel


def _pushes(P, thr, sel):
    pushed = {}
    for s, vs in enumerate(sel):
        for v in vs:
            dv = np.float32(((P[s] - P[v]) ** 2).sum())
            if v > s or not (dv <= thr[v]):
                key = (min(s, v), max(s, v))
                pushed[key] = pushed.get(key, 0) + 1
    return pushed


def _cloud(rng, n, G, clusters):
    c = rng.random((clusters, 3))
    P = np.clip(c[rng.integers(0, clusters, n)] + rng.normal(0, 0.02, (n, 3)), 0, 1 - 1e-12)
    vox = np.floor(P * G).astype(np.int64)
    return P, vox


def _check(P, vox, n, trial, dense):
    bucket = [set() for _ in range(n)]  # symmetric stand-in worksets
    r = random.Random(trial)
    for _ in range(3 * n):
        a, b = r.randrange(n), r.randrange(n)
        if a != b and np.abs(vox[a] - vox[b]).max() <= 1:
            bucket[a].add(b)
            bucket[b].add(a)
    for K in (1, 4, 16):
        thr, sel = _selections(P, vox, K, bucket)
        pushed = _pushes(P, thr, sel)
        union = {(min(s, v), max(s, v)) for s, vs in enumerate(sel) for v in vs}
        assert union, "the clouds must have several points per voxel"
        # never twice (so both worksets get each pair once), never outside
        # the selections, never a pair the worksets already hold
        assert all(c == 1 for c in pushed.values())
        assert set(pushed) <= union
        assert all(b not in bucket[a] for a, b in pushed)
        if not dense:  # no cap binds: every selected pair goes in
            assert set(pushed) == union


def test_no_pair_pushed_twice_and_none_lost_without_caps():
    rng = np.random.default_rng(7)
    for trial in range(4):
        # about two points per voxel: no voxel run or block reaches its cap
        P = rng.random((4000, 3)) * 0.25
        vox = np.floor(P * 56).astype(np.int64)
        counts = {}
        for v in map(tuple, vox):
            counts[v] = counts.get(v, 0) + 1
        assert max(counts.values()) <= 16
        _check(P, vox, len(P), trial, dense=False)


def test_no_pair_pushed_twice_in_dense_voxels():
    rng = np.random.default_rng(8)
    for trial in range(4):
        # dozens of points per voxel: the caps bind and a pair one side never
        # gathered can be left to splaying, but none is pushed twice
        P, vox = _cloud(rng, 1500, 24, 4)
        _check(P, vox, len(P), trial, dense=True)
