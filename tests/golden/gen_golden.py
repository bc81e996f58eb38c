"""Generates the predicate known-answer fixtures in tests/golden/.

Run in a container where the reference sources are mounted; it builds the
reference's own predicate code with `make -C oracle ref` (host predicates.c and
the device predicate headers compiled for the host) and records the signs it
returns:

  orient3d_kat.npz   Common/predicates.c orient3d (host, REAL_TYPE_DOUBLE)
  insphere_kat.npz   Common/predicates.c insphere (host, REAL_TYPE_DOUBLE)
  orient4_kat.npz    GDelPredDevice.h orientation4SoS (insphereexact + 49-depth SoS)

Inputs are seeded: random points, small-lattice points (many exact
degeneracies: coplanar, cospherical, collinear, equal coordinates) and
Pythagorean-triple points on a common sphere.

    python tests/golden/gen_golden.py
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(REPO, "oracle", "_ref")


def _build_ref():
    subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref"])


def _gen_points(rng, n, k):
    """n sets of k points (n, k, 3) mixing generic and degenerate families."""
    out = np.empty((n, k, 3))
    trip = np.array([(3, 4, 0), (0, 3, 4), (4, 0, 3), (0, 0, 5), (5, 0, 0), (0, 5, 0),
                     (3, 0, 4), (4, 3, 0), (0, 4, 3)], dtype=np.float64)
    for i in range(n):
        fam = i % 6
        if fam == 0:
            p = rng.random((k, 3))
        elif fam == 1:
            p = rng.integers(0, 4, size=(k, 3)) / 4.0
        elif fam == 2:
            p = rng.integers(0, 2, size=(k, 3)) / 2.0
        elif fam == 3:
            t = trip[rng.integers(0, len(trip), size=k)]
            s = rng.choice([-1.0, 1.0], size=(k, 3))
            p = 0.5 + s * t / 20.0
        elif fam == 4:
            base = rng.integers(0, 3, size=3) / 2.0
            d = rng.integers(-2, 3, size=3) / 4.0
            t = rng.integers(-3, 4, size=k)[:, None]
            p = base + t * d
            p[: k // 2, 2] += rng.integers(0, 2, size=k // 2) / 8.0
        else:
            p = np.empty((k, 3))
            p[:, 0] = 0.25
            p[:, 1] = rng.integers(0, 5, size=k) / 8.0
            p[:, 2] = rng.integers(0, 2, size=k) / 8.0
        out[i] = p
    return out


def main():
    _build_ref()
    host = ctypes.CDLL(os.path.join(REF, "libref_hostpred.so"))
    dev = ctypes.CDLL(os.path.join(REF, "libref_devpred.so"))
    host.exactinit()
    host.orient3d.restype = ctypes.c_double
    host.insphere.restype = ctypes.c_double
    dev.ref_orient4_sos.restype = ctypes.c_int
    D = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(20240601)

    def distinct(p):
        return len({tuple(r) for r in p}) == len(p)

    # orient3d
    pts = _gen_points(rng, 6000, 4)
    keep = [i for i in range(len(pts)) if distinct(pts[i])]
    pts = np.ascontiguousarray(pts[keep])
    sg = np.empty(len(pts), np.int8)
    for i, p in enumerate(pts):
        a = np.ascontiguousarray(p).ravel()
        ptr = [a[3 * j:].ctypes.data_as(D) for j in range(4)]
        sg[i] = np.sign(host.orient3d(*ptr))
    np.savez_compressed(os.path.join(HERE, "orient3d_kat.npz"), points=pts, sign=sg)

    # insphere
    pts = _gen_points(rng, 6000, 5)
    keep = [i for i in range(len(pts)) if distinct(pts[i])]
    pts = np.ascontiguousarray(pts[keep])
    sg = np.empty(len(pts), np.int8)
    for i, p in enumerate(pts):
        a = np.ascontiguousarray(p).ravel()
        ptr = [a[3 * j:].ctypes.data_as(D) for j in range(5)]
        sg[i] = np.sign(host.insphere(*ptr))
    np.savez_compressed(os.path.join(HERE, "insphere_kat.npz"), points=pts, sign=sg)

    # orient4 with SoS (point indices are the SoS ranks)
    pts = _gen_points(rng, 9000, 5)
    keep = [i for i in range(len(pts)) if distinct(pts[i])]
    pts = np.ascontiguousarray(pts[keep])
    idx = np.stack([rng.choice(1 << 20, size=5, replace=False) for _ in range(len(pts))]).astype(np.int32)
    sg = np.empty(len(pts), np.int8)
    for i in range(len(pts)):
        a = np.ascontiguousarray(pts[i]).ravel()
        ia = np.ascontiguousarray(idx[i])
        sg[i] = dev.ref_orient4_sos(a.ctypes.data_as(D), ia.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    np.savez_compressed(os.path.join(HERE, "orient4_kat.npz"), points=pts, idx=idx, sign=sg)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    sys.exit(main())
