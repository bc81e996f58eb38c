"""Parity of the CUDA path with the oracle, through the C ABI. Needs a B200.

Bit-exact: the canonical tetrahedron list (sorted vertex ids per tet, tets
sorted) and the canonical adjacency must equal the oracle's, which is pinned
to the reference's own predicate code and certified by the validator.
"""
import os

import numpy as np
import pytest

from gstar4d_b200 import workloads

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def tri():
    import gstar4d_b200
    t = gstar4d_b200.Triangulator(do_check=1)
    yield t
    t.close()


def _canon(oracle, tets):
    import gstar4d_b200
    return oracle.canonical(gstar4d_b200.tets_as_array(tets))


def test_device_predicates_match_reference_kat(tri):
    d = np.load(os.path.join(GOLD, "orient3d_kat.npz"))
    got = tri.eval_predicates(0, d["points"].reshape(len(d["sign"]), 12))
    assert np.array_equal(got, d["sign"])
    d = np.load(os.path.join(GOLD, "orient4_kat.npz"))
    got = tri.eval_predicates(1, d["points"].reshape(len(d["sign"]), 15), d["idx"])
    assert np.array_equal(got, d["sign"])
    d = np.load(os.path.join(GOLD, "insphere_kat.npz"))
    got = tri.eval_predicates(2, d["points"].reshape(len(d["sign"]), 15))
    assert np.array_equal(got, d["sign"])


@pytest.mark.parametrize("kind,n,G", [("uniform", 2000, 32), ("uniform", 20000, 64), ("mixed", 20000, 128),
                                      ("degenerate", 20000, 128)])
def test_parity_small_clouds(tri, oracle, kind, n, G):
    pts = {"uniform": workloads.uniform, "mixed": workloads.mixed, "degenerate": workloads.degenerate}[kind](
        n, seed=5)
    tri.config.grid_size = G
    import gstar4d_b200
    with gstar4d_b200.Triangulator(grid_size=G, do_check=1) as t:
        tets, order, stats = t.triangulate(pts, want_order=True)
    ref, ref_order, _ = oracle.triangulate(pts, G)
    assert np.array_equal(order, ref_order), "Morton order differs"
    g, r = _canon(oracle, tets), oracle.canonical(ref)
    assert np.array_equal(g[0], r[0]), "tetrahedra differ"
    assert np.array_equal(g[1], r[1]), "adjacency differs"
    assert stats["tets"] == len(ref)


def test_parity_uniform_100k_full_size(oracle):
    """The 100,000-point uniform configuration at its own grid (256^3)."""
    import gstar4d_b200
    pts, G = workloads.config_cloud("uniform100k")
    with gstar4d_b200.Triangulator(grid_size=G) as t:
        tets, _, stats = t.triangulate(pts)
    ref, _, _ = oracle.triangulate(pts, G)
    g, r = _canon(oracle, tets), oracle.canonical(ref)
    assert np.array_equal(g[0], r[0]) and np.array_equal(g[1], r[1])


def test_parity_degenerate500k_with_large_stars(oracle):
    """The 500,000-point degenerate configuration (sphere + lattice + uniform,
    grid 512^3): stars next to the dense sphere sheet outgrow the small storage
    class and finish in the large class; the result stays bit-exact, exact
    predicates and Simulation of Simplicity included."""
    import gstar4d_b200
    pts, G = workloads.config_cloud("degenerate500k")
    with gstar4d_b200.Triangulator(grid_size=G, do_check=1) as t:
        tets, _, stats = t.triangulate(pts)
    assert stats["large_stars"] > 0
    assert stats["exact_predicates"] > 0
    ref, _, _ = oracle.triangulate(pts, G)
    g, r = _canon(oracle, tets), oracle.canonical(ref)
    assert np.array_equal(g[0], r[0]), "tetrahedra differ"
    assert np.array_equal(g[1], r[1]), "adjacency differs"


def test_parity_dense_voxels_overflow_worksets(oracle):
    """Tight clusters on a coarse grid: dozens of points share a voxel, so the
    voxel leaders' initial worksets overflow their 64 slots; the overflowing
    entries must still reach both points (symmetric worksets), or splaying
    stops with inconsistent stars."""
    import gstar4d_b200
    pts = workloads.clustered(30000, k=4, sigma=0.03, seed=9, uniform_frac=0.1)
    with gstar4d_b200.Triangulator(grid_size=64, do_check=1) as t:
        tets, _, _ = t.triangulate(pts)
    ref, _, _ = oracle.triangulate(pts, 64)
    g, r = _canon(oracle, tets), oracle.canonical(ref)
    assert np.array_equal(g[0], r[0]), "tetrahedra differ"
    assert np.array_equal(g[1], r[1]), "adjacency differs"


def _clustered_dense(k):
    import gstar4d_b200
    pts = workloads.clustered(120000, k=16, sigma=0.01, seed=12)
    os.environ["G4D_BLOCK_K"] = str(k)
    try:
        with gstar4d_b200.Triangulator(grid_size=128, do_check=1) as t:
            tets, _, st = t.triangulate(pts)
    finally:
        del os.environ["G4D_BLOCK_K"]
    return pts, tets, st


@pytest.mark.parametrize("k", [1, 64])
def test_block_pairs_leave_the_triangulation_unchanged(oracle, k):
    """Workset pairs from 3x3x3 voxel blocks (the G4D_BLOCK_K nearest block
    points of every point whose voxel holds several points) only change
    splaying's work: a clustered cloud with several points in many voxels
    triangulates as the oracle does for any K."""
    pts, tets, st = _clustered_dense(k)
    ref, _, _ = oracle.triangulate(pts, 128)
    g, r = _canon(oracle, tets), oracle.canonical(ref)
    assert np.array_equal(g[0], r[0]), "tetrahedra differ"
    assert np.array_equal(g[1], r[1]), "adjacency differs"
    assert st["block_pairs"] > 0


def test_block_pairs_save_splaying_work(oracle):
    """The default K against none: the same triangulation, fewer insertions
    left to splaying."""
    pts, tets0, st0 = _clustered_dense(0)
    _, tets, st = _clustered_dense(16)
    assert st0["block_pairs"] == 0 and st["block_pairs"] > 0
    a, b = _canon(oracle, tets0), _canon(oracle, tets)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert st["splay_insertions"] < 0.8 * st0["splay_insertions"]


def test_morton_index_space_and_gdel_entry_points(oracle):
    """gdelInit/gdelCompute/getTetraFromGpu shape: points already in grid units,
    overwritten with the Morton order; output in Morton indices."""
    import gstar4d_b200
    G = 64
    rng = np.random.default_rng(8)
    pts = 1.0 + (G - 3) * rng.random((3000, 3))
    orig = pts.copy()
    with gstar4d_b200.Triangulator(grid_size=G) as t:
        work = pts.copy()
        t.gdel_init(work)
        t.gdel_compute()
        tets = t.get_tetra_from_gpu()
        t.gdel_deinit()
    # points came back sorted: a permutation of the input
    assert sorted(map(tuple, work)) == sorted(map(tuple, orig))
    # tets index the returned (sorted) array; generic points make the SoS ranks
    # irrelevant, so the oracle on the same array must agree
    ref, _, _ = oracle.triangulate(work, G)
    g, r = _canon(oracle, tets), oracle.canonical(ref)
    assert np.array_equal(g[0], r[0])


@pytest.mark.parametrize("kind,n,G", [("mixed", 20000, 64), ("uniform", 100000, 256), ("clustered", 50000, 128)])
def test_voronoi_grid_is_exact(tri, oracle, kind, n, G):
    """Every voxel's PBA site is at the exact minimum squared distance."""
    pts = {"mixed": workloads.mixed, "uniform": workloads.uniform, "clustered": workloads.clustered}[kind](n, seed=6)
    sites = tri.voronoi(pts, G)
    _, vox = oracle.morton_order(pts, G)
    ref = oracle.edt(vox, G)
    g = np.arange(G)
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    sx, sy, sz = (sites & 1023).astype(np.int64), ((sites >> 10) & 1023).astype(np.int64), ((sites >> 20) & 1023).astype(np.int64)
    d_gpu = (sx - X.ravel()) ** 2 + (sy - Y.ravel()) ** 2 + (sz - Z.ravel()) ** 2
    rv = vox[ref].astype(np.int64)
    d_ref = (rv[:, 0] - X.ravel()) ** 2 + (rv[:, 1] - Y.ravel()) ** 2 + (rv[:, 2] - Z.ravel()) ** 2
    assert (sites != 0xFFFFFFFF).all()
    assert np.array_equal(d_gpu, d_ref)
    # every site is an occupied voxel
    occ = set((vox[:, 0] | (vox[:, 1] << 10) | (vox[:, 2] << 20)).tolist())
    assert set(np.unique(sites).tolist()) <= occ


def test_invalid_arguments_raise(tri):
    import gstar4d_b200
    with pytest.raises(gstar4d_b200.G4DError) as e:
        tri.triangulate(np.random.default_rng(1).random((4, 3)))
    assert e.value.status == 1
    with pytest.raises(gstar4d_b200.G4DError):
        with gstar4d_b200.Triangulator(grid_size=48) as t:
            t.triangulate(np.random.default_rng(1).random((100, 3)))


def test_tiny_clouds_pump_and_match(oracle):
    import gstar4d_b200
    for n in (5, 9, 64):
        pts = workloads.uniform(n, seed=n)
        with gstar4d_b200.Triangulator(grid_size=32) as t:
            tets, _, _ = t.triangulate(pts)
        ref, _, _ = oracle.triangulate(pts, 32)
        g, r = _canon(oracle, tets), oracle.canonical(ref)
        assert np.array_equal(g[0], r[0]) and np.array_equal(g[1], r[1]), n


def test_float32_points_match_the_widened_double_path(tri, oracle):
    """g4d_triangulate_to_f32 (the reference's default float RealType): the
    same tetrahedra and adjacency as the double path on the widened values,
    and as the oracle."""
    pts32 = workloads.mixed(30000, seed=12).astype(np.float32)
    _, first = np.unique(pts32, axis=0, return_index=True)
    pts32 = np.ascontiguousarray(pts32[np.sort(first)])
    a, _, _ = tri.triangulate(pts32)
    b, _, _ = tri.triangulate(pts32.astype(np.float64))
    ga, gb = _canon(oracle, a), _canon(oracle, b)
    assert np.array_equal(ga[0], gb[0]) and np.array_equal(ga[1], gb[1])
    ref, _, _ = oracle.triangulate(pts32.astype(np.float64), 256)
    r = oracle.canonical(ref)
    assert np.array_equal(ga[0], r[0]) and np.array_equal(ga[1], r[1])


@pytest.mark.parametrize("name", ["mixed1m", "clustered8m"])
def test_voronoi_exact_at_full_size_sampled(tri, oracle, name):
    """The digital Voronoi diagram of the 1M (512^3) and 8M (1024^3)
    configurations: on 2M sampled voxels the site is an occupied voxel at the
    exact minimum squared distance (nearest occupied voxel by a k-d tree over
    all of them; squared distances of integer points are compared as
    integers)."""
    from scipy.spatial import cKDTree
    pts, G = workloads.config_cloud(name)
    sites = tri.voronoi(pts, G)
    _, vox = oracle.morton_order(pts, G)
    occ = np.unique(vox.astype(np.int64), axis=0)
    rng = np.random.default_rng(17)
    idx = rng.integers(0, G ** 3, 2_000_000)
    q = np.stack([idx % G, (idx // G) % G, idx // (G * G)], axis=1)
    _, nn = cKDTree(occ).query(q)
    d_ref = ((occ[nn] - q) ** 2).sum(axis=1)
    s = sites[idx].astype(np.int64)
    assert (s != 0xFFFFFFFF).all()
    sv = np.stack([s & 1023, (s >> 10) & 1023, (s >> 20) & 1023], axis=1)
    assert np.array_equal(((sv - q) ** 2).sum(axis=1), d_ref)
    codes = set((occ[:, 0] | (occ[:, 1] << 10) | (occ[:, 2] << 20)).tolist())
    assert all(int(c) in codes for c in np.unique(s))


@pytest.mark.parametrize("form", [0, 1, 2])
def test_every_pba_form_gives_the_same_triangulation(oracle, monkeypatch, form):
    """The per-width tuner may pick any of the PBA pass forms (one thread per
    line, or lines staged in shared memory in two tile shapes); each one gives
    exact distances (test_voronoi_grid_is_exact covers the tuned one) and the
    same triangulation."""
    import gstar4d_b200
    pts = workloads.clustered(40000, seed=23)
    monkeypatch.setenv("G4D_PBA_FORM", str(form))
    with gstar4d_b200.Triangulator(grid_size=128) as t:
        sites = t.voronoi(pts, 128)
        tets, _, _ = t.triangulate(pts)
    _, vox = oracle.morton_order(pts, 128)
    ref = oracle.edt(vox, 128)
    g = np.arange(128)
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    s = sites.astype(np.int64)
    d = (s & 1023) - X.ravel(), ((s >> 10) & 1023) - Y.ravel(), ((s >> 20) & 1023) - Z.ravel()
    rv = vox[ref].astype(np.int64)
    dr = rv[:, 0] - X.ravel(), rv[:, 1] - Y.ravel(), rv[:, 2] - Z.ravel()
    assert np.array_equal(sum(c * c for c in d), sum(c * c for c in dr))
    r, _, _ = oracle.triangulate(pts, 128)
    a, b = _canon(oracle, tets), oracle.canonical(r)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
