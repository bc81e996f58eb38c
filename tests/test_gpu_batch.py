"""Batched triangulation (g4d_triangulate_batch) against one call per cloud and
against the oracle. Needs a B200.

Every cloud of a batch must come back bit-exact: the same canonical
tetrahedra and adjacency, in cloud-local input indices, as the same cloud
triangulated alone at the same grid width.
"""
import numpy as np
import pytest

from gstar4d_b200 import workloads

pytestmark = pytest.mark.gpu


def auto_grid(n):
    g = 32
    while g ** 3 < 134 * n and g < 1024:
        g *= 2
    return g


def _batch(count, seed, hi):
    sizes = workloads.batch_sizes(count, seed=seed, hi=hi)
    clouds = [workloads.batch_cloud(int(n), kind=i % 3, seed=seed * 1000 + i) for i, n in enumerate(sizes)]
    offs = np.zeros(len(clouds) + 1, np.int64)
    offs[1:] = np.cumsum([len(c) for c in clouds])
    return clouds, np.concatenate(clouds), offs


def _canon(oracle, tets):
    import gstar4d_b200
    return oracle.canonical(gstar4d_b200.tets_as_array(tets))


def test_batch_matches_single_cloud_calls(oracle):
    import gstar4d_b200
    clouds, pts, offs = _batch(48, seed=3, hi=6000)
    with gstar4d_b200.Triangulator() as t:
        tets, toffs, stats = t.triangulate_batch(pts, offs)
        assert len(toffs) == len(clouds) + 1 and toffs[-1] == len(tets)
        for c, cloud in enumerate(clouds):
            single, _, _ = t.triangulate(cloud)
            got = _canon(oracle, tets[toffs[c]:toffs[c + 1]])
            exp = _canon(oracle, single)
            assert np.array_equal(got[0], exp[0]), "cloud %d: tetrahedra differ" % c
            assert np.array_equal(got[1], exp[1]), "cloud %d: adjacency differs" % c
    # a few clouds against the oracle itself
    for c in (0, 7, 20):
        ref, _, _ = oracle.triangulate(clouds[c], auto_grid(len(clouds[c])))
        got = _canon(oracle, tets[toffs[c]:toffs[c + 1]])
        exp = oracle.canonical(ref)
        assert np.array_equal(got[0], exp[0]) and np.array_equal(got[1], exp[1]), c


def test_batch_fixed_grid_and_repeat_calls(oracle):
    """All clouds on one grid width (one stack), and a second call on the same
    context reusing its buffers."""
    import gstar4d_b200
    clouds, pts, offs = _batch(12, seed=4, hi=3000)
    with gstar4d_b200.Triangulator(grid_size=64) as t:
        a, ao, _ = t.triangulate_batch(pts, offs)
        b, bo, _ = t.triangulate_batch(pts, offs)
    assert np.array_equal(ao, bo)
    for c in range(len(clouds)):
        ref, _, _ = oracle.triangulate(clouds[c], 64)
        for tets, toffs in ((a, ao), (b, bo)):
            got = _canon(oracle, tets[toffs[c]:toffs[c + 1]])
            exp = oracle.canonical(ref)
            assert np.array_equal(got[0], exp[0]) and np.array_equal(got[1], exp[1]), c


def test_batch_autotuned_grids_match_single_calls(oracle):
    """grid_size -1: the batch tunes a width per (size bucket, distribution
    class); single calls on the same context reuse those widths, so every
    cloud must still match its single-call result; the device-resident batch
    gives the same tetrahedra."""
    import torch
    import gstar4d_b200
    clouds, pts, offs = _batch(40, seed=5, hi=20000)
    with gstar4d_b200.Triangulator(grid_size=-1) as t:
        tets, toffs, _ = t.triangulate_batch(pts, offs)
        d_pts = torch.from_numpy(pts).cuda()
        dptr, ntet, doffs, _ = t.triangulate_batch_device(d_pts.data_ptr(), offs)
        assert ntet == len(tets) and np.array_equal(doffs, toffs)
        view = type("DeviceTets", (), {"__cuda_array_interface__": {
            "shape": (ntet, 8), "typestr": "<i4", "data": (dptr, False), "version": 3}})()
        dev = torch.as_tensor(view, device="cuda").cpu().numpy()
        for c in range(len(clouds)):
            # tetrahedron numbering follows the splaying's atomic order: compare canonical forms
            got = oracle.canonical(dev[toffs[c]:toffs[c + 1]])
            exp = _canon(oracle, tets[toffs[c]:toffs[c + 1]])
            assert np.array_equal(got[0], exp[0]) and np.array_equal(got[1], exp[1]), c
        for c, cloud in enumerate(clouds):
            single, _, _ = t.triangulate(cloud)
            got = _canon(oracle, tets[toffs[c]:toffs[c + 1]])
            exp = _canon(oracle, single)
            assert np.array_equal(got[0], exp[0]) and np.array_equal(got[1], exp[1]), c


def test_batch_rejects_tiny_cloud():
    import gstar4d_b200
    pts = np.random.default_rng(1).random((20, 3))
    with gstar4d_b200.Triangulator() as t:
        with pytest.raises(gstar4d_b200.G4DError) as e:
            t.triangulate_batch(pts, np.array([0, 3, 20], np.int64))
    assert e.value.status == 1


def test_batch_into_pinned_buffer_over_many_passes(oracle, monkeypatch):
    """g4d_triangulate_batch_to: results copied into a caller (pinned) buffer
    pass by pass while later passes compute; passes limited to 20k points so
    the batch takes several. Every cloud must match the library-allocated
    batch; a buffer one tetrahedron short is refused with the count set."""
    import torch
    import gstar4d_b200
    monkeypatch.setenv("G4D_WAVE_POINTS", "20000")
    clouds, pts, offs = _batch(30, seed=8, hi=9000)
    with gstar4d_b200.Triangulator(grid_size=64) as t:
        ref, ref_offs, _ = t.triangulate_batch(pts, offs)
        buf = torch.empty((len(ref) + 16, 8), dtype=torch.int32).pin_memory()
        out = buf.numpy().view(gstar4d_b200.TET_DTYPE).reshape(-1)
        got, got_offs, _ = t.triangulate_batch(pts, offs, out=out)
        assert np.array_equal(got_offs, ref_offs) and len(got) == len(ref)
        for c in range(len(clouds)):
            a = _canon(oracle, got[got_offs[c]:got_offs[c + 1]])
            b = _canon(oracle, ref[ref_offs[c]:ref_offs[c + 1]])
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), c
        short = out[: len(ref) - 1]
        with pytest.raises(gstar4d_b200.G4DError) as e:
            t.triangulate_batch(pts, offs, out=short)
        assert e.value.status == 1


def test_batch_of_64_clouds_from_the_4096_generator_matches_oracle(oracle):
    """The first 64 clouds of the 4,096-cloud benchmark generator (sizes
    log-uniform up to 50,000; uniform, Gaussian and 8-cluster clouds), batched
    at the reference's density rule and with autotuned widths, every cloud
    compared with the oracle. The clouds are in general position, so the
    triangulation does not depend on the grid width the tuner picks."""
    import gstar4d_b200
    sizes = workloads.batch_sizes(4096, seed=1)[:64]
    kinds = np.random.default_rng(1 + 7).integers(0, 3, size=4096)[:64]
    clouds = [workloads.batch_cloud(int(n), int(k), 1 * 100003 + i) for i, (n, k) in enumerate(zip(sizes, kinds))]
    assert max(len(c) for c in clouds) > 20000
    offs = np.zeros(len(clouds) + 1, np.int64)
    offs[1:] = np.cumsum([len(c) for c in clouds])
    pts = np.concatenate(clouds)
    refs = [oracle.canonical(oracle.triangulate(c, auto_grid(len(c)))[0]) for c in clouds]
    for grid in (0, -1):
        with gstar4d_b200.Triangulator(grid_size=grid) as t:
            if grid < 0:
                t.triangulate_batch(pts, offs)  # the first call tunes the widths
            tets, toffs, _ = t.triangulate_batch(pts, offs)
        for c in range(len(clouds)):
            got = _canon(oracle, tets[toffs[c]:toffs[c + 1]])
            assert np.array_equal(got[0], refs[c][0]), "grid %d, cloud %d: tetrahedra differ" % (grid, c)
            assert np.array_equal(got[1], refs[c][1]), "grid %d, cloud %d: adjacency differs" % (grid, c)
