"""The static error bound of the filter-only star insertions, checked on the CPU.

The filter-only insertion kernels (gstar4d_b200/csrc/g4d_star.cu, warp_insert)
compare the lifted determinant of four coordinates relative to the star's
point with orient4_static_bound(R) (gstar4d_b200/csrc/g4d_predicates.cuh),
where R is the largest magnitude among the star's cached coordinates, instead
of the per-call bound 32 * 2^-53 * perm. This restates the determinant and
its permanent as orient4_filter_rel computes them and checks, with exact
rational arithmetic:

  - perm <= 72 R^5 for every input whose coordinates are at most R, including
    the extreme sign patterns, so the static bound is never below the per-call
    one (the shipped constant covers 32 * 72 * 2^-53 and the rounding of R^5);
  - wherever the double-precision determinant clears the static bound, its
    sign is the exact sign, on random and on nearly cospherical inputs (the
    star's point and the four points on one sphere, then moved by a few ulps).
    Python rounds every operation; the device may fuse a multiply and an add,
    which rounds once instead of twice and so stays within the same bound.
"""
import itertools
import math
import random
from fractions import Fraction

CONST = 2.5606e-13  # orient4_static_bound's constant
EPS = 2.0 ** -53


def _static_bound(r):
    r2 = r * r
    b = CONST * (r2 * r2 * r)
    return math.inf if b < 1e-250 else b


def _parts(a, b, c, d, F=float):
    """det and perm of orient4_filter_rel (rows a, b, c, d relative to the star)."""
    aex, aey, aez = map(F, a)
    bex, bey, bez = map(F, b)
    cex, cey, cez = map(F, c)
    dex, dey, dez = map(F, d)
    aexbey, bexaey = aex * bey, bex * aey
    bexcey, cexbey = bex * cey, cex * bey
    cexdey, dexcey = cex * dey, dex * cey
    dexaey, aexdey = dex * aey, aex * dey
    aexcey, cexaey = aex * cey, cex * aey
    bexdey, dexbey = bex * dey, dex * bey
    ab, bc, cd = aexbey - bexaey, bexcey - cexbey, cexdey - dexcey
    da, ac, bd = dexaey - aexdey, aexcey - cexaey, bexdey - dexbey
    abP, bcP = abs(aexbey) + abs(bexaey), abs(bexcey) + abs(cexbey)
    cdP, daP = abs(cexdey) + abs(dexcey), abs(dexaey) + abs(aexdey)
    acP, bdP = abs(aexcey) + abs(cexaey), abs(bexdey) + abs(dexbey)
    abc = aez * bc - bez * ac + cez * ab
    bcd = bez * cd - cez * bd + dez * bc
    cda = cez * da + dez * ac + aez * cd
    dab = dez * ab + aez * bd + bez * da
    abcP = abs(aez) * bcP + abs(bez) * acP + abs(cez) * abP
    bcdP = abs(bez) * cdP + abs(cez) * bdP + abs(dez) * bcP
    cdaP = abs(cez) * daP + abs(dez) * acP + abs(aez) * cdP
    dabP = abs(dez) * abP + abs(aez) * bdP + abs(bez) * daP
    alift = aex * aex + aey * aey + aez * aez
    blift = bex * bex + bey * bey + bez * bez
    clift = cex * cex + cey * cey + cez * cez
    dlift = dex * dex + dey * dey + dez * dez
    det = (dlift * abc - clift * dab) + (blift * cda - alift * bcd)
    perm = (dlift * abcP + clift * dabP) + (blift * cdaP + alift * bcdP)
    return det, perm


def _rmax(*pts):
    return max(abs(v) for p in pts for v in p)


def test_constant_covers_the_per_call_bound():
    assert Fraction(CONST) >= Fraction(32 * 72) * Fraction(EPS) * (1 + 8 * Fraction(EPS))


def test_permanent_at_most_72_r5():
    rng = random.Random(3)
    R = 1.75
    # every coordinate at +-R: the permanent's largest values
    for signs in itertools.islice(itertools.product((-1, 1), repeat=12), 0, 4096, 7):
        pts = [tuple(R * s for s in signs[3 * i:3 * i + 3]) for i in range(4)]
        _, perm = _parts(*pts, F=Fraction)
        assert perm <= 72 * Fraction(R) ** 5
    for _ in range(2000):
        r = rng.choice((1e-3, 0.5, 3.0, 1e4))
        pts = [tuple(rng.uniform(-r, r) for _ in range(3)) for _ in range(4)]
        _, perm = _parts(*pts, F=Fraction)
        assert perm <= 72 * Fraction(_rmax(*pts)) ** 5


def _exact_sign(pts):
    det, _ = _parts(*pts, F=Fraction)
    return (det > 0) - (det < 0)


def _check(pts, r):
    det, _ = _parts(*pts)
    bound = _static_bound(r)
    if det > bound:
        assert _exact_sign(pts) == 1
        return 1
    if -det > bound:
        assert _exact_sign(pts) == -1
        return 1
    return 0


def test_decided_signs_are_exact_random():
    rng = random.Random(5)
    decided = 0
    for _ in range(3000):
        pts = [tuple(rng.uniform(-1.0, 1.0) for _ in range(3)) for _ in range(4)]
        # the star's other cached points may be farther: R at least this set's own
        r = _rmax(*pts) * rng.choice((1.0, 1.0, 2.0))
        decided += _check(pts, r)
    assert decided > 2500  # generic inputs are decided by the filter


def test_decided_signs_are_exact_near_cospherical():
    rng = random.Random(6)
    decided = 0
    n = 4000
    for _ in range(n):
        # a sphere through the star's point (the origin), four points on it,
        # then every coordinate moved by a relative amount between a few ulps
        # and 1e-4, so that the cases fall on both sides of the bound
        c = [rng.uniform(-1.0, 1.0) for _ in range(3)]
        rad = math.sqrt(sum(v * v for v in c))
        scale = 10.0 ** -rng.uniform(4.0, 16.0)
        pts = []
        for _ in range(4):
            u = [rng.gauss(0.0, 1.0) for _ in range(3)]
            nu = math.sqrt(sum(v * v for v in u))
            p = [c[k] + rad * u[k] / nu for k in range(3)]
            p = [v * (1.0 + scale * rng.uniform(-1.0, 1.0)) + rng.randint(-2, 2) * math.ulp(v) for v in p]
            pts.append(tuple(p))
        decided += _check(pts, _rmax(*pts))
    assert 0.2 * n < decided < 0.95 * n  # both decided and undecided cases occur
