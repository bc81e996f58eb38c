"""Host-side steps of the path pinned to the reference's own code, compiled
here by `make -C oracle ref` (oracle/_ref/libref_app.so; skipped where the
reference sources were not available to build it). CPU only.

  - point generation for the command line: g4d_make_points against
    Application::makePoints + DtRandom (Main/Application.cpp:316-473,
    Common/DtRandom.cpp:44-109), byte-equal for all five distributions;
  - the Morton order that defines the SoS ranks: the oracle's order (which the
    GPU order equals, tests/test_gpu_parity.py) against the reference's
    GetMortonNumber (GDelaunay/GDelData.cu:51-87) and a stable sort by it;
  - file input: the command line's reading and scaling against readPoints and
    _scalePoint (Main/Application.cpp:475-603).
"""
import ctypes
import os

import numpy as np
import pytest

from gstar4d_b200 import workloads

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_APP = os.path.join(REPO, "oracle", "_ref", "libref_app.so")

pytestmark = pytest.mark.skipif(not os.path.exists(REF_APP), reason="reference host code not built here")


@pytest.fixture(scope="module")
def ref():
    R = ctypes.CDLL(REF_APP)
    vp = ctypes.c_void_p
    R.ref_make_points.argtypes = [ctypes.c_int] * 4 + [vp]
    R.ref_read_points.argtypes = [ctypes.c_char_p, ctypes.c_int, vp, ctypes.c_int]
    R.ref_scale_value.argtypes = [ctypes.c_double, ctypes.c_float, ctypes.c_float, ctypes.c_double]
    R.ref_scale_value.restype = ctypes.c_double
    R.ref_morton_keys.argtypes = [vp, ctypes.c_int, vp]
    return R


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("dist", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("n,grid,seed", [(30000, 256, 0), (5000, 64, 1), (20000, 512, -3)])
def test_generated_points_equal_reference(ref, dist, n, grid, seed):
    from gstar4d_b200 import api
    want = np.empty((n, 3))
    assert ref.ref_make_points(n, dist, grid, seed, _p(want)) == n
    got = api.make_points(n, grid, dist, seed)
    assert got.tobytes() == want.tobytes()


def _ref_order(ref, vox):
    keys = np.empty(len(vox), np.int32)
    ref.ref_morton_keys(_p(np.ascontiguousarray(vox, dtype=np.float64)), len(vox), _p(keys))
    # thrust::sort_by_key on int keys is a stable radix sort
    return np.argsort(keys, kind="stable").astype(np.int32)


@pytest.mark.parametrize("name", ["uniform100k", "mixed1m", "degenerate500k"])
def test_morton_order_equals_reference(oracle, ref, name):
    pts, G = workloads.config_cloud(name, scale=0.25 if name != "uniform100k" else 1.0)
    order, vox = oracle.morton_order(pts, G)  # vox in sorted order
    vox_in = np.empty_like(vox)
    vox_in[order] = vox
    # the reference's key of a grid point is that of its voxel (it truncates)
    assert np.array_equal(order, _ref_order(ref, vox_in))
    # and of the scaled points themselves: the voxel is the truncation
    assert (vox >= 1).all() and (vox <= G - 2).all()


def test_morton_order_of_cli_points_in_grid_units(oracle, ref):
    """Generated points are already in grid units: no scaling, Morton keys of
    the coordinates themselves (the gdelInit path of the command line)."""
    from gstar4d_b200 import api
    for dist in range(5):
        pts = api.make_points(20000, 128, dist, 5)
        keys = np.empty(len(pts), np.int32)
        ref.ref_morton_keys(_p(pts), len(pts), _p(keys))
        order = np.argsort(keys, kind="stable")
        q = pts.astype(np.int64)
        mine = np.zeros(len(pts), np.int64)
        for b in range(10):
            for c in range(3):
                mine |= ((q[:, c] >> b) & 1) << (3 * b + c)
        assert np.array_equal(np.argsort(mine, kind="stable"), order)


def test_scale_value_equals_reference(ref):
    from gstar4d_b200 import __main__ as cli
    rng = np.random.default_rng(9)
    for grid in (64, 256, 1024):
        for lo, hi in ((-3.7, 12.25), (0.0, 1.0), (1e-3, 7e4)):
            v = np.concatenate([rng.uniform(lo, hi, 3000), [lo, hi]]).astype(np.float32)
            mn, mx = np.float32(v.min()), np.float32(v.max())
            pts = v.astype(np.float64)[: len(v) // 3 * 3].reshape(-1, 3)
            got = cli.scale_points(pts, grid, mn, mx)
            want = np.array([[ref.ref_scale_value(float(grid), float(mn), float(mx), float(c)) for c in p]
                             for p in pts])
            assert got.tobytes() == np.ascontiguousarray(want).tobytes()


def test_read_points_equals_reference(ref, tmp_path):
    from gstar4d_b200 import __main__ as cli
    rng = np.random.default_rng(10)
    pts = rng.normal(5.0, 3.0, (4000, 3))
    pts[100:110] = pts[:10]  # duplicates the reader drops
    f = tmp_path / "pts.txt"
    with open(f, "w") as fh:
        for p in pts:
            fh.write("%.9g %.9g %.9g\n" % tuple(p))
    for grid in (128, 512):
        want = np.empty((len(pts), 3))
        m = ref.ref_read_points(str(f).encode(), grid, _p(want), len(pts))
        raw, mn, mx, dup = cli.read_point_file(str(f))
        got = cli.scale_points(raw, grid, mn, mx)
        assert dup == 10 and m == len(got)
        assert got.tobytes() == np.ascontiguousarray(want[:m]).tobytes()


REF_APP_F32 = os.path.join(REPO, "oracle", "_ref", "libref_app_f32.so")


@pytest.fixture(scope="module")
def ref32():
    if not os.path.exists(REF_APP_F32):
        pytest.skip("float build of the reference host code not built here")
    R = ctypes.CDLL(REF_APP_F32)
    vp = ctypes.c_void_p
    R.ref_make_points.argtypes = [ctypes.c_int] * 4 + [vp]
    R.ref_read_points.argtypes = [ctypes.c_char_p, ctypes.c_int, vp, ctypes.c_int]
    R.ref_scale_value.argtypes = [ctypes.c_double, ctypes.c_float, ctypes.c_float, ctypes.c_double]
    R.ref_scale_value.restype = ctypes.c_double
    return R


def test_float_build_file_input_equals_reference(ref32, tmp_path):
    """The default float build (RealType = float) scales file input in float
    arithmetic; the command line's -float mode must give its scaled points."""
    from gstar4d_b200 import __main__ as cli
    rng = np.random.default_rng(11)
    pts = np.concatenate([rng.normal(-2.0, 40.0, (3000, 3)), rng.random((1000, 3))])
    f = tmp_path / "pts.txt"
    with open(f, "w") as fh:
        for p in pts:
            fh.write("%.8g %.8g %.8g\n" % tuple(p))
    for grid in (64, 256, 1024):
        want = np.empty((len(pts), 3))
        m = ref32.ref_read_points(str(f).encode(), grid, _p(want), len(pts))
        raw, mn, mx, _ = cli.read_point_file(str(f))
        got = cli.scale_points(raw, grid, mn, mx, as_float=True)
        assert m == len(got)
        assert got.tobytes() == np.ascontiguousarray(want[:m]).tobytes()
        # and the double build differs in general (the scaling rounds differently)
        dbl = cli.scale_points(raw, grid, mn, mx)
        assert not np.array_equal(dbl, got)


def test_float_build_generates_the_same_points(ref, ref32):
    for dist in range(5):
        a = np.empty((3000, 3))
        b = np.empty((3000, 3))
        ref.ref_make_points(3000, dist, 128, 2, _p(a))
        ref32.ref_make_points(3000, dist, 128, 2, _p(b))
        assert a.tobytes() == b.tobytes()
