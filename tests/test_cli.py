"""The command line's host logic (flags, point generators, file input, PLY
output, adjacency check). CPU only."""
import numpy as np
import pytest

from gstar4d_b200 import __main__ as cli


def test_flags_follow_the_reference():
    o = cli.parse_args(["-n", "5000", "-g", "128", "-s", "7", "-r", "2", "-d", "3", "-check", "-timing", "-stats",
                        "-verbose", "-sort", "-predThreadNum", "64", "-predBlockNum", "8"])
    assert (o["n"], o["grid"], o["seed"], o["run_num"], o["dist"]) == (5000, 128, 7, 2, 3)
    assert o["check"] and o["timing"] and o["stats"] and o["verbose"]
    assert o["facet_max"] == 10000000  # Main.cpp default for non-uniform distributions
    assert cli.parse_args([])["facet_max"] == 12000000
    with pytest.raises(ValueError):
        cli.parse_args(["-bogus"])
    with pytest.raises(ValueError):
        cli.parse_args(["-d", "9"])
    assert cli.parse_args(["-h"])["help"]


@pytest.mark.parametrize("dist", range(5))
def test_generators_give_distinct_points_in_grid_units(dist):
    p = cli.make_points(4000, 64, dist, seed=3)
    assert p.shape == (4000, 3)
    assert p.min() >= 1.0 and p.max() <= 62.0
    assert len(np.unique(p, axis=0)) == len(p)
    assert np.array_equal(p, cli.make_points(4000, 64, dist, seed=3))


def test_read_points_drops_duplicates(tmp_path):
    f = tmp_path / "pts.txt"
    # a flat stream of coordinates, three per point; a trailing partial point is ignored
    f.write_text("0 0 0\n1 2 3\n0 0 0\n4 5 6 7\n")
    p = cli.read_points(str(f))
    assert p.tolist() == [[0, 0, 0], [1, 2, 3], [4, 5, 6]]


def test_ply_layout_and_adjacency_check(tmp_path):
    from gstar4d_b200.api import TET_DTYPE
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], float)
    t = np.zeros(2, TET_DTYPE)
    t["v"] = [[0, 1, 2, 3], [1, 2, 3, 4]]
    t["opp"] = [[1, -1, -1, -1], [-1, -1, -1, 0]]
    assert cli.check_adjacency(t) == 0
    t["opp"][0, 0] = -1
    assert cli.check_adjacency(t) == 1
    f = tmp_path / "m.ply"
    cli.write_ply(str(f), pts, t)
    lines = f.read_text().splitlines()
    assert lines[0] == "ply" and "element vertex 5" in lines and "element face 6" in lines
    assert lines[lines.index("end_header") + 6] == "3 0 1 2"


def test_float_flag_rounds_points_to_float32(tmp_path):
    """-float: the reference's default float build reads and holds float32
    coordinates; the points become those values (as doubles), and points the
    rounding makes equal are dropped."""
    assert cli.parse_args(["-float"])["float"] and not cli.parse_args([])["float"]
    f = tmp_path / "pts.txt"
    f.write_text("0.1 0.2 0.3\n0.10000000001 0.2 0.3\n1 2 3\n")
    p = cli.read_points(str(f), as_float=True)
    assert p.dtype == np.float64 and len(p) == 2
    assert np.array_equal(p[0], np.array([0.1, 0.2, 0.3], np.float32).astype(np.float64))
    g = cli.as_float_values(cli.make_points(2000, 64, 0, seed=1))
    assert np.array_equal(g, g.astype(np.float32).astype(np.float64))
