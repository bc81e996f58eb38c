"""The 64-bit-limb exact lifted orientation (gstar4d_b200/csrc/g4d_exact64.cuh),
compiled for the host, against Python's arbitrary-precision integers.

The device predicates use this routine for the exact sign whenever the
rescaled coordinates are below 2^61 (the common case of the exact path), so
its widths and carries are checked here on random, clustered, exactly
degenerate (cocircular rectangles and integer spheres, with and without a
unit perturbation) and extreme inputs. The sign convention is the reference's
lifted 5x5 determinant translated by the last point (orient4,
GDelaunay/GDelPredDevice.h:115-135): det [D_r | |D_r|^2] over D_r = p_r - p_4.
"""
import os
import random
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "gstar4d_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include "g4d_exact64.cuh"
int main() {
    long long v[15];
    for (;;) {
        for (int i = 0; i < 15; ++i)
            if (scanf("%lld", &v[i]) != 1) return 0;
        int64_t X[5][3];
        for (int i = 0; i < 5; ++i)
            for (int c = 0; c < 3; ++c) X[i][c] = v[3 * i + c];
        if (!g4d::x64::fits61(X)) { printf("W\n"); continue; }
        printf("%d\n", g4d::x64::orient4_sign(X));
    }
}
"""

LIM = (1 << 61) - 1


def _det(m):
    if len(m) == 1:
        return m[0][0]
    s = 0
    for c, v in enumerate(m[0]):
        if v:
            s += (-1) ** c * v * _det([row[:c] + row[c + 1:] for row in m[1:]])
    return s


def _sign(p):
    D = [[p[r][c] - p[4][c] for c in range(3)] for r in range(4)]
    v = _det([d + [d[0] * d[0] + d[1] * d[1] + d[2] * d[2]] for d in D])
    return (v > 0) - (v < 0)


def _cases(rng, n):
    out = []
    for _ in range(n):  # full range
        out.append([[rng.randint(-LIM, LIM) for _ in range(3)] for _ in range(5)])
    for _ in range(n):  # clustered about a large centre
        c = [rng.randint(-LIM // 2, LIM // 2) for _ in range(3)]
        sp = rng.choice([1, 10, 1 << 20, 1 << 40, 1 << 58])
        out.append([[c[k] + rng.randint(-sp, sp) for k in range(3)] for _ in range(5)])
    while len(out) < 3 * n:  # a rectangle in a plane and any fifth point: exactly zero
        s = rng.choice([1, 3, 1 << 30, 1 << 55])
        x1, x2, y1, y2, z = (rng.randint(-1000, 1000) for _ in range(5))
        sh = [rng.randint(-(1 << 59), 1 << 59) for _ in range(3)]
        pts = [[x1, y1, z], [x2, y1, z], [x1, y2, z], [x2, y2, z], [rng.randint(-1000, 1000) for _ in range(3)]]
        rng.shuffle(pts)
        pts = [[sh[k] + s * q[k] for k in range(3)] for q in pts]
        if all(abs(v) <= LIM for q in pts for v in q):
            out.append(pts)
    sphere = {r2: [(a, b, c) for a in range(-14, 15) for b in range(-14, 15) for c in range(-14, 15)
                   if a * a + b * b + c * c == r2] for r2 in (25, 50, 99, 169, 147)}
    for _ in range(n):  # integer points on a sphere, perturbed by 0 or 1 unit
        sols = sphere[rng.choice(list(sphere))]
        s = rng.choice([1, 1 << 20, 1 << 56])
        out.append([[s * v + rng.choice([0, 0, 0, 1, -1]) for v in rng.choice(sols)] for _ in range(5)])
    for _ in range(n // 4):  # extremes
        out.append([[rng.choice([LIM, -LIM, LIM - 1, -LIM + 1, 0, 1, -1]) for _ in range(3)] for _ in range(5)])
    return out


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_exact64_matches_python_integers(tmp_path):
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    subprocess.check_call(["g++", "-O2", "-Wno-unknown-pragmas", "-I", CSRC, "-o", str(exe), str(src)])
    cases = _cases(random.Random(11), 1500)
    inp = "\n".join(" ".join(str(v) for q in p for v in q) for p in cases) + "\n"
    got = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True).stdout.split()
    assert len(got) == len(cases)
    want = [str(_sign(p)) for p in cases]
    bad = [(p, w, g) for p, w, g in zip(cases, want, got) if w != g]
    assert not bad, bad[:3]
    assert want.count("0") > 1000  # the degenerate families reach the zero case


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_exact64_rejects_wide_coordinates(tmp_path):
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    subprocess.check_call(["g++", "-O2", "-Wno-unknown-pragmas", "-I", CSRC, "-o", str(exe), str(src)])
    wide = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1 << 61, 0, 0]]
    inp = " ".join(str(v) for q in wide for v in q) + "\n"
    got = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True).stdout.split()
    assert got == ["W"]  # left to the 32-bit-limb routine
