"""The CPU oracle, pinned against the reference's own predicate code and checked
with the reference's validator rules. CPU only."""
import os

import numpy as np
import pytest

from gstar4d_b200 import workloads

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_orient3d_matches_reference_kat(oracle):
    d = np.load(os.path.join(GOLD, "orient3d_kat.npz"))
    got = np.array([oracle.orient3d(p) for p in d["points"]], np.int8)
    assert (got == d["sign"]).all(), np.flatnonzero(got != d["sign"])[:10]
    assert (d["sign"] == 0).sum() > 100  # the fixture exercises exact zeros


def test_insphere_matches_reference_kat(oracle):
    d = np.load(os.path.join(GOLD, "insphere_kat.npz"))
    got = np.array([oracle.insphere(p) for p in d["points"]], np.int8)
    assert (got == d["sign"]).all(), np.flatnonzero(got != d["sign"])[:10]
    assert (d["sign"] == 0).sum() > 100


def test_orient4_sos_matches_reference_kat(oracle):
    d = np.load(os.path.join(GOLD, "orient4_kat.npz"))
    got = np.array([oracle.orient4_sos(p, i) for p, i in zip(d["points"], d["idx"])], np.int8)
    assert (got == d["sign"]).all(), np.flatnonzero(got != d["sign"])[:10]
    assert (got != 0).all()


def test_orient4_sos_is_antisymmetric(oracle):
    d = np.load(os.path.join(GOLD, "orient4_kat.npz"))
    rng = np.random.default_rng(3)
    for k in range(0, len(d["sign"]), 7):
        p, i = d["points"][k], d["idx"][k]
        perm = rng.permutation(5)
        inv = sum(1 for a in range(5) for b in range(a + 1, 5) if perm[a] > perm[b])
        s = oracle.orient4_sos(p[perm], i[perm])
        assert s == d["sign"][k] * (-1) ** inv


def test_orient4_sos_random_against_reference_build(oracle):
    import ctypes
    oracle.build()  # also builds oracle/_ref when the reference sources are mounted
    path = os.path.join(oracle.REF_DIR, "libref_devpred.so")
    if not os.path.exists(path):
        pytest.skip("reference build unavailable")
    dev = ctypes.CDLL(path)
    rng = np.random.default_rng(11)
    for _ in range(3000):
        p = rng.integers(0, 3, size=(5, 3)) / 2.0
        if len({tuple(r) for r in p}) < 5:
            continue
        idx = rng.choice(100000, size=5, replace=False).astype(np.int32)
        a = np.ascontiguousarray(p).ravel()
        r = dev.ref_orient4_sos(a.ctypes.data_as(ctypes.c_void_p), idx.ctypes.data_as(ctypes.c_void_p))
        assert oracle.orient4_sos(p, idx) == r


def test_morton_order_is_stable_and_sorted(oracle):
    pts = workloads.uniform(5000, seed=4)
    pts[100] = pts[7]  # a duplicate voxel: stable order keeps input order
    order, vox = oracle.morton_order(pts, 64)
    assert sorted(order.tolist()) == list(range(len(pts)))
    assert vox.min() >= 1 and vox.max() <= 64 - 2

    def spread(v):
        out = 0
        for b in range(10):
            out |= ((v >> b) & 1) << (3 * b)
        return out
    keys = [spread(x) | (spread(y) << 1) | (spread(z) << 2) for x, y, z in vox]
    assert all(keys[i] <= keys[i + 1] for i in range(len(keys) - 1))
    for i in range(len(keys) - 1):
        if keys[i] == keys[i + 1]:
            assert order[i] < order[i + 1]


def test_edt_is_exact_nearest_site(oracle):
    G = 32
    pts = workloads.uniform(300, seed=5)
    order, vox = oracle.morton_order(pts, G)
    site = oracle.edt(vox, G)
    g = np.arange(G)
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    d2 = ((coords[:, None, :] - vox[None, :, :]) ** 2).sum(-1)
    best = d2.min(1)
    got = d2[np.arange(len(site)), site]
    assert (got == best).all()


@pytest.mark.parametrize("kind,n,G", [("uniform", 3000, 32), ("mixed", 6000, 64), ("degenerate", 6000, 64)])
def test_oracle_triangulation_validates(oracle, kind, n, G):
    pts = {"uniform": workloads.uniform, "mixed": workloads.mixed, "degenerate": workloads.degenerate}[kind](n, seed=2)
    tets, order, st = oracle.triangulate(pts, G)
    rank = np.empty(len(pts), np.int32)
    rank[order] = np.arange(len(pts), dtype=np.int32)
    rep = oracle.validate(pts, tets, rank)
    assert rep["euler"] == 1
    for k in ("orient_fail", "insphere_fail", "adjacency_asym", "sos_fail"):
        assert rep[k] == 0, (k, rep)
    assert rep["V"] == len(pts)
    assert st["consistency_repairs"] == 0


def test_oracle_is_deterministic_across_threads(oracle):
    pts = workloads.mixed(4000, seed=9)
    a, _, _ = oracle.triangulate(pts, 64, threads=1)
    b, _, _ = oracle.triangulate(pts, 64, threads=8)
    ca, cb = oracle.canonical(a), oracle.canonical(b)
    assert np.array_equal(ca[0], cb[0]) and np.array_equal(ca[1], cb[1])


def test_oracle_grid_size_does_not_change_result(oracle):
    """The tetrahedra depend on coordinates and Morton index order only; two
    grids with the same Morton order must give the same mesh, and any grid must
    give the same vertex sets up to the SoS index relabelling."""
    pts = workloads.uniform(3000, seed=12)
    a, oa, _ = oracle.triangulate(pts, 32)
    b, ob, _ = oracle.triangulate(pts, 64)
    if np.array_equal(oa, ob):
        assert np.array_equal(oracle.canonical(a)[0], oracle.canonical(b)[0])
    # generic points: no exact degeneracy, so the mesh is the plain Delaunay mesh
    assert np.array_equal(oracle.canonical(a)[0], oracle.canonical(b)[0])


def test_mlp_oracle_gradient_matches_finite_differences():
    """The FP64 network restatement (the checker of the tensor-core training
    kernel): analytic gradient of the unrounded function vs central
    differences, on a few coordinates of every parameter block."""
    from oracle import mlp_oracle as mo
    _, x = mo.sample_rows(40, seed=3)
    y = (np.random.default_rng(4).random(40) < 0.5).astype(np.float64)
    p = mo.init_params(seed=5)
    _, g, _ = mo.forward_backward(x, y, p, rounding=False)
    rng = np.random.default_rng(6)
    blocks = [(mo.P_W1, mo.P_B1), (mo.P_B1, mo.P_W2), (mo.P_W2, mo.P_B2), (mo.P_B2, mo.P_W3), (mo.P_W3, mo.P_B3),
              (mo.P_B3, mo.P_W4), (mo.P_W4, mo.P_B4), (mo.P_B4, mo.NPARAMS)]
    for lo, hi in blocks:
        live = [i for i in range(lo, hi) if not (lo == mo.P_W1 and (i - lo) % 16 >= 6)]
        for i in rng.choice(live, size=min(4, len(live)), replace=False):
            h = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[i] += h
            pm[i] -= h
            fd = (mo.forward_backward(x, y, pp, rounding=False)[0] - mo.forward_backward(x, y, pm, rounding=False)[0]) / (2 * h)
            assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (i, fd, g[i])
