"""g4d_voronoi_noalloc (device buffers, fixed library scratch) against
g4d_voronoi (context-allocated buffers) through the C ABI. Needs a B200.

The grids are integer voxel codes, so the tolerance is zero: bit-exact. Two
calls in a row, the second on a smaller grid, show that what the shared scratch
keeps from an earlier call does not leak into the next.
"""
import ctypes

import numpy as np
import pytest

from gstar4d_b200 import workloads

pytestmark = pytest.mark.gpu


def _noalloc(lib, pts, grid):
    import torch
    d_xyz = torch.from_numpy(np.ascontiguousarray(pts, dtype=np.float64)).cuda()
    d_sites = torch.empty(grid ** 3, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    st = lib.g4d_voronoi_noalloc(ctypes.c_void_p(d_xyz.data_ptr()), len(pts), grid,
                                 ctypes.c_void_p(d_sites.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert st == 0, lib.g4d_status_string(st)
    stream.synchronize()
    return d_sites.cpu().numpy().view(np.uint32)


def test_noalloc_voronoi_matches_context_entry_two_calls():
    import gstar4d_b200
    from gstar4d_b200 import api
    lib = api.load()
    clouds = [(workloads.uniform(200000, seed=11), 128), (workloads.mixed(20000, seed=12), 64)]
    got = [_noalloc(lib, pts, G) for pts, G in clouds]
    with gstar4d_b200.Triangulator() as t:
        for (pts, G), g in zip(clouds, got):
            ref = t.voronoi(pts, G)
            assert (g != 0xFFFFFFFF).all()
            assert np.array_equal(g, ref)


def test_noalloc_rejects_sizes_beyond_scratch():
    import torch
    from gstar4d_b200 import api
    lib = api.load()
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    # n and grid beyond the fixed scratch: G4D_ERR_CAPACITY, nothing enqueued
    assert lib.g4d_voronoi_noalloc(ctypes.c_void_p(d.data_ptr()), (1 << 18) + 1, 64,
                                   ctypes.c_void_p(d.data_ptr()), None) == 6
    assert lib.g4d_voronoi_noalloc(ctypes.c_void_p(d.data_ptr()), 100, 256,
                                   ctypes.c_void_p(d.data_ptr()), None) == 6
    assert lib.g4d_voronoi_noalloc(None, 100, 64, ctypes.c_void_p(d.data_ptr()), None) == 1
