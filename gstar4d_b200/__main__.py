"""Command line with the reference's flags (GDelaunay/Main/Main.cpp:40-207,
Application.cpp:213-603):

    python -m gstar4d_b200 [-n PointNum] [-g GridSize] [-s Seed] [-r RunNum]
                           [-d Distribution] [-f FacetMax] [-verbose] [-stats]
                           [-timing] [-check] [-inFile F] [-outFile F]
                           [-predThreadNum N] [-predBlockNum N] [-sort]
                           [-proposal WEIGHTS.npy] [-device D] [-float]

Runs follow the reference's Application::doRun / _doRun (Application.cpp:100-307):
per run a "Seed:" line, the points, the gdelInit/gdelCompute facade in the
Morton index space, the Init / PBA / InitStar / Consistency / StarOutput /
Total Time block (milliseconds), -check and -outFile on the Morton-sorted
points, the seed incremented; after the runs one line appended to
gStar4D-time.txt (and to gStar4D-count.txt with -stats) in the reference's CSV
layout, times averaged in seconds. Generated points lie in grid units
[1, G-2] like the reference's makePoints (Application.cpp:316-360); points read
with -inFile are parsed as float values (the reference reads float tokens in
both of its builds), duplicates dropped, and scaled like _scalePoint
(Application.cpp:589-603) in place, so the scaled points are the ones
triangulated, as in the reference. -outFile also writes the input points
(Input-Points.asc, or Input-Scaled-Points.asc for file input). Generated
points are the reference's own: its makePoints and KISS generator (DtRandom,
64-bit `unsigned long` as on Linux) restated in C++ (g4d_make_points), so
`-n -g -d -s` give the same point sets as the reference binary built on Linux.
-f, -predThreadNum and -predBlockNum are accepted and have no effect (no
per-loop facet bound, no fixed exact-predicate thread pool). -proposal loads
learned star-proposal weights (float32[9473], see Triangulator.train_proposal).
-float follows the reference's default RealType = float build
(Common/Geometry.h:53-57): file input is scaled in float arithmetic, so the
scaled points are the float build's (generated points are float values in
both builds); the predicates are exact in both builds, so the triangulation is
that build's.
"""
import sys
import time

import numpy as np

DISTRIBUTIONS = ("Uniform", "Gaussian", "Ball", "Sphere", "Grid")

USAGE = ("Syntax: gstar4d [-n PointNum] [-g GridSize] [-s Seed] [-r Max] [-d Distribution] [-f FacetMax] "
         "[-verbose] [-stats] [-timing] [-check] [-inFile F] [-outFile F] [-proposal W.npy] [-device D] [-float]\n"
         "Distribution: 0 - Uniform, 1 - Gaussian, 2 - Ball, 3 - Sphere, 4 - Grid")


def parse_args(argv):
    """Returns the option dict, or raises ValueError on a bad argument."""
    o = {"seed": 0, "run_num": 1, "grid": 256, "n": 100000, "dist": 0, "facet_max": -1, "verbose": False,
         "stats": False, "timing": False, "check": False, "in_file": None, "out_file": None,
         "pred_thread_num": -1, "pred_block_num": -1, "sort": True, "proposal": None, "device": 0, "help": False,
         "float": False}
    valued = {"-n": ("n", int), "-g": ("grid", int), "-r": ("run_num", int), "-s": ("seed", int),
              "-f": ("facet_max", int), "-d": ("dist", int), "-inFile": ("in_file", str),
              "-outFile": ("out_file", str), "-predThreadNum": ("pred_thread_num", int),
              "-predBlockNum": ("pred_block_num", int), "-proposal": ("proposal", str), "-device": ("device", int)}
    flags = {"-verbose": "verbose", "-stats": "stats", "-timing": "timing", "-check": "check", "-sort": "sort",
             "-float": "float"}
    i = 0
    while i < len(argv):
        a = argv[i]
        if a in valued:
            if i + 1 >= len(argv):
                raise ValueError("missing value for " + a)
            key, conv = valued[a]
            o[key] = conv(argv[i + 1])
            i += 2
            continue
        if a in flags:
            o[flags[a]] = True
        elif a in ("-h", "--help"):
            o["help"] = True
        else:
            raise ValueError("Error in input argument: " + a)
        i += 1
    if not 0 <= o["dist"] < len(DISTRIBUTIONS):
        raise ValueError("distribution must be 0..4")
    if o["facet_max"] == -1:  # Main.cpp: 12M for uniform, else 10M (no effect here)
        o["facet_max"] = 12000000 if o["dist"] == 0 else 10000000
    return o


def make_points(n, grid, dist, seed):
    """The reference's generated points for -n -g -d -s (Application::makePoints
    with DtRandom's KISS numbers, restated in C++ as g4d_make_points): n
    distinct float values in grid units [1, G-2], as float64."""
    from gstar4d_b200 import api
    return api.make_points(n, grid, dist, seed)


def as_float_values(points):
    """Points rounded to float32 (then held as the equal doubles), duplicates
    the rounding creates dropped (first occurrence kept)."""
    p = np.asarray(points, dtype=np.float32).astype(np.float64)
    _, first = np.unique(p, axis=0, return_index=True)
    return np.ascontiguousarray(p[np.sort(first)])


def read_point_file(path):
    """The reference's readPoints (Application.cpp:475-587): whitespace-
    separated tokens parsed as float, three per point, duplicates dropped (first
    occurrence kept). Returns (points as float64 holding the float values, the
    float minimum and maximum over all tokens, number of duplicates)."""
    with open(path) as f:
        vals = np.array(f.read().split(), dtype=np.float32)
    mn = np.float32(vals.min()) if len(vals) else np.float32(0)
    mx = np.float32(vals.max()) if len(vals) else np.float32(0)
    pts = vals[: len(vals) // 3 * 3].astype(np.float64).reshape(-1, 3)
    _, first = np.unique(pts, axis=0, return_index=True)
    keep = np.sort(first)
    return np.ascontiguousarray(pts[keep]), mn, mx, len(pts) - len(keep)


def scale_points(points, grid, mn, mx, as_float=False):
    """_scalePoint (Application.cpp:589-603): v -> (G - 3) (v - min) / (max -
    min) + 1 with the float bounds (their difference taken in float), the rest
    in RealType: double (the REAL_TYPE_DOUBLE build), or float with as_float
    (the default float build, Common/Geometry.h:53-57, where every step rounds
    to float). Duplicates the scaling creates are dropped."""
    f32 = np.float32
    rng = f32(mx) - f32(mn)
    if as_float:
        t = np.asarray(points, np.float64).astype(f32) - f32(mn)
        p = ((f32(grid) - f32(3.0)) * t / rng + f32(1.0)).astype(np.float64)
    else:
        p = (float(grid) - 3.0) * (np.asarray(points, np.float64) - np.float64(mn)) / np.float64(rng) + 1.0
    _, first = np.unique(p, axis=0, return_index=True)
    return np.ascontiguousarray(p[np.sort(first)])


def read_points(path, as_float=False):
    """Whitespace-separated coordinates, three per point, duplicates dropped
    (first occurrence kept); parsed as float32 values with as_float."""
    with open(path) as f:
        vals = np.array(f.read().split(), dtype=np.float32 if as_float else np.float64).astype(np.float64)
    pts = vals[: len(vals) // 3 * 3].reshape(-1, 3)
    _, first = np.unique(pts, axis=0, return_index=True)
    return np.ascontiguousarray(pts[np.sort(first)])


def write_asc(path, points):
    """One point per line, coordinates separated by spaces, printed like the
    reference's default stream formatting (6 significant digits)."""
    with open(path, "w") as f:
        for p in np.asarray(points, np.float64):
            f.write("%g %g %g\n" % (p[0], p[1], p[2]))


def log_lines(o, n, sums):
    """The lines the reference appends to gStar4D-time.txt and
    gStar4D-count.txt (Application.cpp:160-196). sums: per-stage millisecond
    sums over the runs (init, pba, star, splay, out, total) and the insertion
    and loop counters; times are averaged and given in seconds."""
    runs = o["run_num"]
    head = "GridSize,%d,Runs,%d,Points,%d,Input,%s," % (
        o["grid"], runs, n, o["in_file"] if o["in_file"] else DISTRIBUTIONS[o["dist"]])
    sec = lambda k: "%g" % (sums[k] / (runs * 1000.0))
    time_line = head + ("Total Time,%s,Init Time,%s,PBA Time,%s,Star Time,%s,Splay Time,%s,Out Time,%s" % (
        sec("total"), sec("init"), sec("pba"), sec("star"), sec("splay"), sec("out")))
    count_line = head + "Total insertions,%d,Star insertions,%d,Splay insertions,%d,Loop number,%d" % (
        sums["star_ins"] + sums["splay_ins"], sums["star_ins"], sums["splay_ins"], sums["loops"])
    return time_line, count_line


def write_ply(path, points, tets):
    """The reference's TetraMesh::writeToFile (Geometry.cu:396-466): ASCII PLY,
    each vertex as its coordinates in the stream's default format (%g) each
    followed by a space, then three faces per tetrahedron, tetrahedron by
    tetrahedron: (v0 v1 v2), (v0 v1 v3), (v0 v2 v3)."""
    v = np.asarray(tets["v"] if getattr(tets, "dtype", None) is not None and tets.dtype.names else tets)[:, :4]
    with open(path, "w") as f:
        f.write("ply\nformat ascii 1.0\nelement vertex %d\nproperty float x\nproperty float y\nproperty float z\n"
                "element face %d\nproperty list uchar int vertex_index\nend_header\n" % (len(points), 3 * len(v)))
        f.write("".join("%g %g %g \n" % (p[0], p[1], p[2]) for p in np.asarray(points, np.float64)))
        f.write("".join("3 %d %d %d \n3 %d %d %d \n3 %d %d %d \n" % (t[0], t[1], t[2], t[0], t[1], t[3], t[0], t[2], t[3])
                        for t in v.tolist()))


def print_check(rep):
    """The device validator's report in TetraMesh::check's words
    (Common/Geometry.cu:200-393); returns True when the mesh passed."""
    print("Euler Characteristic:")
    print("V: %d E: %d F: %d T: %d Euler: %d" % (rep["vertices"], rep["edges"], rep["triangles"], rep["tets"],
                                                 rep["euler"]))
    if rep["euler"] != 1:
        print("Euler check failed!")
    if rep["orient_fail"]:
        print("Orientation check failed!!!")
        print("Tetra failures: %d" % rep["orient_fail"])
    else:
        print("Tetra orientation is correct!")
    if rep["insphere_fail"]:
        print("In-sphere check failed!!!")
        print("Tetra failures: %d" % rep["insphere_fail"])
    else:
        print("Tetra in-sphere is correct!")
    if rep["adjacency_fail"]:
        print("Adjacency check failed: %d links" % rep["adjacency_fail"])
    return rep["euler"] == 1 and not (rep["orient_fail"] or rep["insphere_fail"] or rep["adjacency_fail"])


def main(argv=None):
    try:
        o = parse_args(sys.argv[1:] if argv is None else argv)
    except ValueError as e:
        print(str(e) + "\n\n" + USAGE)
        return 1
    if o["help"]:
        print(USAGE)
        return 1
    import gstar4d_b200
    weights = np.load(o["proposal"]).astype(np.float32) if o["proposal"] else None
    cfg = dict(grid_size=o["grid"], do_check=int(o["check"]), log_verbose=int(o["verbose"]),
               log_stats=int(o["stats"]), log_timing=int(o["timing"]), device=o["device"],
               facet_max=o["facet_max"], pred_thread_num=o["pred_thread_num"],
               pred_block_num=o["pred_block_num"], proposal=int(weights is not None))
    sums = dict(init=0.0, pba=0.0, star=0.0, splay=0.0, out=0.0, total=0.0, star_ins=0, splay_ins=0, loops=0)
    totals = []
    n_used = o["n"]
    for run in range(o["run_num"]):
        seed = o["seed"] + run
        print("Seed: %d" % seed)
        if o["in_file"]:
            print("Reading from point file ...")
            raw, mn, mx, dups = read_point_file(o["in_file"])
            if dups:
                print("%d duplicate points in input file!" % dups)
            pts = scale_points(raw, o["grid"], mn, mx, as_float=o["float"])
            if o["stats"]:
                print("Min: %g Max: %g Min-Scaled: %g Max-Scaled: %g" % (
                    mn, mx, 1.0, (o["grid"] - 3.0) + 1.0))
            if o["out_file"]:
                write_asc("Input-Scaled-Points.asc", pts)
        else:
            # float values already: the same points in both of the reference's builds
            pts = make_points(o["n"], o["grid"], o["dist"], seed)
            if o["out_file"]:
                write_asc("Input-Points.asc", pts)
        n_used = len(pts)
        work = np.ascontiguousarray(pts, dtype=np.float64).copy()
        with gstar4d_b200.Triangulator(**cfg) as t:
            if weights is not None:
                t.proposal_weights(weights)
            t0 = time.perf_counter()
            t.gdel_init(work)  # sorted in place, like gdelInit
            init_ms = (time.perf_counter() - t0) * 1e3
            times = t.gdel_compute()
            tot_ms = (time.perf_counter() - t0) * 1e3
            tets = t.get_tetra_from_gpu() if o["out_file"] else None
            rep = t.check_mesh() if o["check"] else None
            st = t.stats()
            t.gdel_deinit()
        print("")
        print("Init:        %g" % init_ms)
        print("PBA:         %g" % times[0])
        print("InitStar:    %g" % times[1])
        print("Consistency: %g" % times[2])
        print("StarOutput:  %g" % times[3])
        print("")
        print("Total Time:  %g" % tot_ms)
        for k, v in zip(("init", "pba", "star", "splay", "out", "total"), (init_ms,) + tuple(times) + (tot_ms,)):
            sums[k] += v
        sums["star_ins"] += st["star_insertions"]
        sums["splay_ins"] += st["splay_insertions"]
        sums["loops"] += st["loops"]
        totals.append(tot_ms)
        if o["stats"] or o["verbose"]:
            print("Star insertions: %d  Splay insertions: %d  Loops: %d  Tetra: %d  Exact predicates: %d" % (
                st["star_insertions"], st["splay_insertions"], st["loops"], st["tets"], st["exact_predicates"]))
        if o["check"]:  # star consistency ran on the device during splaying; then the mesh validator
            if not print_check(rep):
                return 2
        if o["out_file"]:
            write_ply(o["out_file"], work, tets)  # the tetrahedra index the Morton-sorted points
    time_line, count_line = log_lines(o, n_used, sums)
    with open("gStar4D-time.txt", "a") as f:
        f.write(time_line + "\n")
    if o["stats"]:
        with open("gStar4D-count.txt", "a") as f:
            f.write(count_line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
