"""The oracle's validator (the reference's checks, Geometry.cu:200-393, plus
adjacency symmetry) rejects meshes with planted mistakes, so a passing
validation means something. Mistakes are planted in oracle output on the CPU.
"""
import numpy as np

from gstar4d_b200 import workloads

FAILS = ("orient_fail", "insphere_fail", "adjacency_asym", "sos_fail")


def _mesh(oracle, n=2000, seed=3):
    pts = workloads.uniform(n, seed=seed)
    tets, order, _ = oracle.triangulate(pts, 32)
    rank = np.empty(len(pts), np.int32)
    rank[order] = np.arange(len(pts), dtype=np.int32)
    return pts, tets, rank


def _ok(rep):
    return rep["euler"] == 1 and all(rep[k] == 0 for k in FAILS)


def test_unchanged_mesh_passes(oracle):
    pts, tets, rank = _mesh(oracle)
    assert _ok(oracle.validate(pts, tets, rank))


def test_flipped_tetrahedron_is_caught(oracle):
    pts, tets, rank = _mesh(oracle)
    bad = tets.copy()
    interior = np.flatnonzero((bad[:, 4:] >= 0).all(axis=1))[0]
    bad[interior, [0, 1]] = bad[interior, [1, 0]]  # orientation reversed
    bad[interior, [4, 5]] = bad[interior, [5, 4]]  # adjacency kept consistent with the swap
    rep = oracle.validate(pts, bad, rank)
    assert rep["orient_fail"] > 0


def test_broken_adjacency_is_caught(oracle):
    pts, tets, rank = _mesh(oracle)
    bad = tets.copy()
    t = np.flatnonzero((bad[:, 4:] >= 0).all(axis=1))[0]
    bad[t, 4] = next(k for k in range(len(bad)) if k not in (t, bad[t, 4]))  # a wrong neighbour
    assert oracle.validate(pts, bad, rank)["adjacency_asym"] > 0


def test_missing_tetrahedron_is_caught(oracle):
    pts, tets, rank = _mesh(oracle)
    t = np.flatnonzero((tets[:, 4:] >= 0).all(axis=1))[-1]
    keep = np.ones(len(tets), bool)
    keep[t] = False
    remap = np.full(len(tets), -1, np.int64)
    remap[keep] = np.arange(keep.sum())
    bad = tets[keep].copy()
    opp = bad[:, 4:].astype(np.int64)
    bad[:, 4:] = np.where(opp >= 0, remap[np.clip(opp, 0, None)], -1).astype(np.int32)
    assert not _ok(oracle.validate(pts, bad, rank))


def _two_tets(oracle, pts, a, b, c, d, e):
    """Tetrahedra (a,b,c,d) and (a,b,c,e) glued along abc, oriented as the
    reference requires (orient3d <= 0)."""
    out = []
    for apex in (d, e):
        v = [a, b, c, apex]
        if oracle.orient3d(pts[v]) > 0:
            v[0], v[1] = v[1], v[0]
        out.append(v)
    tets = np.full((2, 8), -1, np.int32)
    for k, v in enumerate(out):
        tets[k, :4] = v
        tets[k, 4 + 3] = 1 - k  # the face abc is opposite the apex (position 3)
    return tets


def test_non_delaunay_face_is_caught(oracle):
    # a triangle with two apexes close to its plane: the point below lies inside
    # the circumsphere of the tetrahedron above, so the two-tetrahedron mesh
    # (valid, but not Delaunay) must fail the empty-sphere test, while the
    # oracle's own mesh of the same points (three tetrahedra about the edge de)
    # passes.
    pts = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0],
                    [0.3, 0.3, 0.1], [0.3, 0.3, -0.1]]) * 0.5 + 0.25
    rank = np.arange(5, dtype=np.int32)
    bad = _two_tets(oracle, pts, 0, 1, 2, 3, 4)
    rep = oracle.validate(pts, bad, rank)
    assert rep["euler"] == 1 and rep["orient_fail"] == 0 and rep["adjacency_asym"] == 0
    assert rep["insphere_fail"] > 0

    tets, order, _ = oracle.triangulate(pts, 32)
    rank[order] = np.arange(5, dtype=np.int32)
    assert len(tets) == 3
    assert _ok(oracle.validate(pts, tets, rank))


def test_delaunay_two_tetrahedra_pass(oracle):
    # the same triangle with far apexes: the two-tetrahedron mesh is Delaunay
    pts = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0],
                    [0.3, 0.3, 1.0], [0.3, 0.3, -1.0]]) * 0.25 + 0.4
    rank = np.arange(5, dtype=np.int32)
    good = _two_tets(oracle, pts, 0, 1, 2, 3, 4)
    assert _ok(oracle.validate(pts, good, rank))
