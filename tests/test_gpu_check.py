"""The device validator (g4d_check_mesh / g4d_check_tets, the reference's
TetraMesh::check of Common/Geometry.cu:200-393 on the GPU) against the
oracle's validator. Needs a B200.

Its counts (V, E, F, T) must equal the oracle's on the library's own meshes,
and meshes with mistakes planted on the host copy (reversed orientation, a
wrong neighbour, a missing tetrahedron, a valid but non-Delaunay pair) must
fail it like they fail the oracle. Every planted index stays inside the
arrays' bounds.
"""
import numpy as np
import pytest

from gstar4d_b200 import workloads

pytestmark = pytest.mark.gpu


def _oracle_counts(oracle, pts, tets):
    order, _ = oracle.morton_order(pts, 64)
    rank = np.empty(len(pts), np.int32)
    rank[order] = np.arange(len(pts), dtype=np.int32)
    return oracle.validate(pts, tets, rank)


@pytest.mark.parametrize("kind,n,G", [("mixed", 20000, 64), ("degenerate", 20000, 128), ("clustered", 30000, 64)])
def test_validator_passes_library_meshes_with_oracle_counts(oracle, kind, n, G):
    import gstar4d_b200
    pts = {"mixed": workloads.mixed, "degenerate": workloads.degenerate,
           "clustered": workloads.clustered}[kind](n, seed=41)
    with gstar4d_b200.Triangulator(grid_size=G) as t:
        tets, _, _ = t.triangulate(pts)
        rep = t.check_mesh()
        # the gdel facade (points in grid units, output in Morton indices)
        work = 1.0 + (G - 3) * pts
        t.gdel_init(work)
        t.gdel_compute()
        rep_morton = t.check_mesh()
        nt_morton = len(t.get_tetra_from_gpu())
    arr = gstar4d_b200.tets_as_array(tets)
    ref = _oracle_counts(oracle, pts, arr)
    assert rep["euler"] == 1
    assert rep["orient_fail"] == 0 and rep["insphere_fail"] == 0 and rep["adjacency_fail"] == 0
    assert (rep["vertices"], rep["edges"], rep["triangles"], rep["tets"]) == (ref["V"], ref["E"], ref["F"], ref["T"])
    assert rep_morton["euler"] == 1 and rep_morton["tets"] == nt_morton
    assert rep_morton["orient_fail"] == rep_morton["insphere_fail"] == rep_morton["adjacency_fail"] == 0


def _mesh(oracle):
    pts = workloads.uniform(2000, seed=3)
    tets, _, _ = oracle.triangulate(pts, 32)
    return pts, tets


def test_validator_catches_planted_mistakes(oracle):
    import gstar4d_b200
    pts, tets = _mesh(oracle)
    interior = np.flatnonzero((tets[:, 4:] >= 0).all(axis=1))
    with gstar4d_b200.Triangulator() as t:
        good = t.check_tets(pts, tets)
        assert good["euler"] == 1 and good["orient_fail"] == good["insphere_fail"] == good["adjacency_fail"] == 0

        flipped = tets.copy()
        k = interior[0]
        flipped[k, [0, 1]] = flipped[k, [1, 0]]
        flipped[k, [4, 5]] = flipped[k, [5, 4]]
        assert t.check_tets(pts, flipped)["orient_fail"] > 0

        wrong = tets.copy()
        k = interior[1]
        wrong[k, 4] = next(j for j in range(len(wrong)) if j not in (k, wrong[k, 4]))
        assert t.check_tets(pts, wrong)["adjacency_fail"] > 0

        k = interior[-1]
        keep = np.ones(len(tets), bool)
        keep[k] = False
        remap = np.full(len(tets), -1, np.int64)
        remap[keep] = np.arange(keep.sum())
        missing = tets[keep].copy()
        opp = missing[:, 4:].astype(np.int64)
        missing[:, 4:] = np.where(opp >= 0, remap[np.clip(opp, 0, None)], -1).astype(np.int32)
        rep = t.check_tets(pts, missing)
        assert rep["euler"] != 1 or rep["adjacency_fail"] > 0

        # two tetrahedra on a triangle whose apexes lie close to its plane:
        # valid, not Delaunay
        five = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0],
                         [0.3, 0.3, 0.1], [0.3, 0.3, -0.1]]) * 0.5 + 0.25
        pair = np.full((2, 8), -1, np.int32)
        for j, apex in enumerate((3, 4)):
            v = [0, 1, 2, apex]
            if oracle.orient3d(five[v]) > 0:
                v[0], v[1] = v[1], v[0]
            pair[j, :4] = v
            pair[j, 7] = 1 - j
        rep = t.check_tets(five, pair)
        assert rep["euler"] == 1 and rep["orient_fail"] == 0 and rep["adjacency_fail"] == 0
        assert rep["insphere_fail"] > 0
