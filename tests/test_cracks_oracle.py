"""The oracle's crack initialisers (VFCracks.c, VFCommon.c:823-857) on the CPU:
geometric known answers of the rectangular-crack distance, the AT profiles, and the
several-crack minimum."""
import math

import numpy as np
import pytest

SQUARE = [1, 1, 2, 3, 1, 2, 1, 3, 2]  # P1, P2, P3 of the square [1,3]^2 in the plane z = 2


@pytest.mark.parametrize("x,d", [
    ((2, 2, 2), 0.0),                      # the center: the reference's NaN path -> |s|
    ((2, 2, 2.5), 0.5),                    # above the crack
    ((1.5, 2.5, 1.8), 0.2),                # above an inner point
    ((4, 2, 2.5), math.hypot(1.0, 0.5)),   # beyond the X1 side
    ((2, 4.5, 1), math.hypot(1.5, 1.0)),   # beyond the Y1 side
    ((0, 2, 2), 1.0),                      # in-plane, beyond the X0 side
    ((4, 4, 2), math.sqrt(2.0)),           # along the diagonal: the corner distance
])
def test_rect_distance_known_answers(oracle_mod, x, d):
    o = oracle_mod.Oracle((5, 5, 5), (4, 4, 4), E=1, nu=0.2, Gc=1, epsilon=0.5, eta=1e-8)
    assert o.rect_distance(x, SQUARE) == pytest.approx(d, abs=1e-12)


def test_rect_crack_profiles(oracle_mod):
    """AT1: d/eps (1 - d/(4 eps)) within 2 eps of the crack after removing half the
    thickness; AT2: 0 within the full thickness, else 1 - exp(-d/(2 eps)) of the raw d."""
    n, L, eps, th = (9, 9, 9), (4, 4, 4), 0.5, 0.2
    for atnum in (1, 2):
        o = oracle_mod.Oracle(n, L, E=1, nu=0.2, Gc=1, epsilon=eps, eta=1e-8, atnum=atnum)
        v = o.rect_v(SQUARE, th)
        xs = np.linspace(0, 4, 9)
        Z, Y, X = np.meshgrid(xs, xs, xs, indexing="ij")
        d = np.array([o.rect_distance(p, SQUARE) for p in zip(X.ravel(), Y.ravel(), Z.ravel())])
        if atnum == 1:
            dd = d - th / 2
            ref = np.where(dd <= 0, 0.0, np.where(dd < 2 * eps, dd / eps * (1 - .25 * dd / eps), 1.0))
        else:
            ref = np.where(d <= th, 0.0, 1 - np.exp(-d / 2 / eps))
        assert np.abs(v - ref).max() <= 1e-15


def test_cracks_minimum(oracle_mod):
    o = oracle_mod.Oracle((17, 17, 17), (4, 4, 4), E=1, nu=0.2, Gc=1, epsilon=0.5, eta=1e-8,
                          atnum=1)
    p1 = (2.0, 2.0, 2.0, 0.8, 0.0, 0.0, 0.0)
    p2 = (1.5, 2.5, 2.0, 0.6, 30.0, 60.0, 0.1)
    r1 = SQUARE + [0.0]
    v = o.cracks_v(pennies=[p1, p2], rects=[r1])
    ref = np.minimum(np.minimum(o.penny_v(p1[:3], *p1[3:]), o.penny_v(p2[:3], *p2[3:])),
                     o.rect_v(SQUARE, 0.0))
    assert np.array_equal(v, ref)
    assert np.array_equal(o.cracks_v(), np.ones(o.N))
    # a zero-radius penny contributes nothing
    assert np.array_equal(o.cracks_v(pennies=[(2, 2, 2, 0.0, 0, 0, 0)]), np.ones(o.N))
