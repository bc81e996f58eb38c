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


def test_ply_layout_and_check_report(tmp_path, capsys):
    from gstar4d_b200.api import TET_DTYPE
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], float)
    t = np.zeros(2, TET_DTYPE)
    t["v"] = [[0, 1, 2, 3], [1, 2, 3, 4]]
    t["opp"] = [[1, -1, -1, -1], [-1, -1, -1, 0]]
    ok = dict(vertices=5, edges=9, triangles=7, tets=2, euler=1, orient_fail=0, insphere_fail=0, adjacency_fail=0)
    assert cli.print_check(ok)
    assert "Tetra in-sphere is correct!" in capsys.readouterr().out
    assert not cli.print_check(dict(ok, insphere_fail=3))
    assert "In-sphere check failed!!!" in capsys.readouterr().out
    f = tmp_path / "m.ply"
    cli.write_ply(str(f), pts, t)
    lines = f.read_text().splitlines()
    assert lines[0] == "ply" and "element vertex 5" in lines and "element face 6" in lines
    h = lines.index("end_header")
    # TetraMesh::writeToFile: "x y z " per vertex, three faces per tetrahedron in turn
    assert lines[h + 1] == "0 0 0 " and lines[h + 5] == "1 1 1 "
    assert lines[h + 6:h + 12] == ["3 0 1 2 ", "3 0 1 3 ", "3 0 2 3 ", "3 1 2 3 ", "3 1 2 4 ", "3 1 3 4 "]


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
    g = cli.as_float_values(cli.make_points(2000, 64, 0, seed=1) * 1.1)
    assert np.array_equal(g, g.astype(np.float32).astype(np.float64))


def test_file_input_is_read_as_float_and_scaled_like_the_reference(tmp_path):
    """readPoints + _scalePoint (Application.cpp:475-603): float tokens, the
    bounds over all tokens, duplicates dropped, v -> (G-3)(v-min)/(max-min)+1."""
    f = tmp_path / "pts.txt"
    f.write_text("0.1 2 3\n4 5 6\n0.1 2 3\n-1 0.5 7\n")
    raw, mn, mx, dups = cli.read_point_file(str(f))
    assert dups == 1 and len(raw) == 3
    assert mn == np.float32(-1) and mx == np.float32(7)
    assert raw[0, 0] == float(np.float32(0.1))
    s = cli.scale_points(raw, 64, mn, mx)
    assert s.min() >= 1.0 and s.max() <= 62.0
    assert np.isclose(s[2, 0], 1.0) and np.isclose(s[2, 2], 62.0)


def test_log_lines_follow_the_reference_layout(tmp_path):
    o = cli.parse_args(["-g", "256", "-r", "2", "-d", "1", "-n", "1000"])
    sums = dict(init=2.0, pba=4.0, star=6.0, splay=8.0, out=2.0, total=22.0, star_ins=30, splay_ins=5, loops=7)
    t, c = cli.log_lines(o, 1000, sums)
    assert t == ("GridSize,256,Runs,2,Points,1000,Input,Gaussian,Total Time,0.011,Init Time,0.001,"
                 "PBA Time,0.002,Star Time,0.003,Splay Time,0.004,Out Time,0.001")
    assert c == ("GridSize,256,Runs,2,Points,1000,Input,Gaussian,Total insertions,35,Star insertions,30,"
                 "Splay insertions,5,Loop number,7")
    p = tmp_path / "a.asc"
    cli.write_asc(str(p), np.array([[1.5, 2.0, 1234567.0]]))
    assert p.read_text() == "1.5 2 1.23457e+06\n"
