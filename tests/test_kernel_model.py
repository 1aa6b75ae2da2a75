"""CPU check of the U-apply kernel's schedule (tiling, seams, carries) and modal
element arithmetic, replayed in Python against the oracle."""
import numpy as np
import pytest

import kernel_model as km


def test_modal_element_matches_element_matrix(oracle_mod):
    rng = np.random.default_rng(3)
    o = oracle_mod.Oracle((2, 2, 2), (0.3, 0.5, 0.7), E=2.0, nu=0.3, eta=1e-3)
    lam, mu = 2.0 * 0.3 / 1.3 / 0.4, 2.0 / 1.3 * 0.5
    for _ in range(4):
        v, x = rng.uniform(0, 1, 8), rng.standard_normal(24)
        yref = o.u_element_matrix(0, 0, 0, v) @ x
        for f in (km.u_element, km.u_element_points, km.u_element_sums):
            y = f(x.reshape(8, 3), v, lam, mu, 1e-3, (0.3, 0.5, 0.7)).reshape(24)
            assert np.abs(y - yref).max() <= 1e-14 * np.abs(yref).max()


def test_modal_sum_element_cubic(oracle_mod):
    """The cubic-cell variant of the sum-mode element (every 1/h in the row weight)."""
    rng = np.random.default_rng(4)
    h = 0.25
    o = oracle_mod.Oracle((2, 2, 2), (h, h, h), E=2.0, nu=0.3, eta=1e-3)
    lam, mu = 2.0 * 0.3 / 1.3 / 0.4, 2.0 / 1.3 * 0.5
    for _ in range(4):
        v, x = rng.uniform(0, 1, 8), rng.standard_normal(24)
        yref = o.u_element_matrix(0, 0, 0, v) @ x
        for cubic in (False, True):
            y = km.u_element_sums(x.reshape(8, 3), v, lam, mu, 1e-3, (h, h, h), cubic=cubic)
            assert np.abs(y.reshape(24) - yref).max() <= 1e-14 * np.abs(yref).max()


@pytest.mark.parametrize("h", [(0.3, 0.5, 0.7), (0.25, 0.25, 0.25)])
def test_constant_phase_field_element(oracle_mod, h):
    """Elements whose 8 nodal v are equal: the fixed-weight form (exact cell averages of
    the polynomial stress moments) against the reference's 27-point element matrix."""
    rng = np.random.default_rng(6)
    eta = 1e-3
    o = oracle_mod.Oracle((2, 2, 2), h, E=2.0, nu=0.3, eta=eta)
    lam, mu = 2.0 * 0.3 / 1.3 / 0.4, 2.0 / 1.3 * 0.5
    for vc in (1.0, 0.37, 0.0):
        v = np.full(8, vc)
        x = rng.standard_normal(24)
        yref = o.u_element_matrix(0, 0, 0, v) @ x
        for cubic in ((False, True) if h[0] == h[1] == h[2] else (False,)):
            y = km.u_element_const(x.reshape(8, 3), vc * vc + eta, lam, mu, h, cubic=cubic)
            assert np.abs(y.reshape(24) - yref).max() <= 1e-14 * np.abs(yref).max(), (vc, cubic)


@pytest.mark.parametrize("n,TY,zc", [((37, 21, 13), 8, 5), ((34, 10, 7), 4, 3), ((3, 2, 4), 8, 2)])
def test_tiled_schedule_matches_oracle(oracle_mod, n, TY, zc):
    rng = np.random.default_rng(sum(n))
    o = oracle_mod.Oracle(n, (1.1, 0.9, 0.7), E=3.0, nu=0.2, eta=1e-2)
    lam, mu = 3.0 * 0.2 / 1.2 / 0.6, 3.0 / 1.2 * 0.5
    v, x = rng.uniform(0, 1, o.N), rng.standard_normal(3 * o.N)
    mask, _ = o.bc(oracle_mod.rollers_face())
    bits = (mask.reshape(o.N, 3) * np.array([1, 2, 4])).sum(1).astype(np.uint8)
    yref = o.u_apply(v, x, mask)
    h = tuple(L / (k - 1) for L, k in zip((1.1, 0.9, 0.7), n))
    y = km.u_apply_tiled(x, v, bits, n, h, lam, mu, 1e-2, TY=TY, zc=zc)
    assert np.abs(y - yref).max() <= 1e-13 * np.abs(yref).max()


@pytest.mark.parametrize("n,TY,ncta", [((37, 21, 13), 8, 7), ((34, 10, 7), 4, 5), ((3, 2, 4), 8, 3),
                                       ((37, 21, 13), 8, 1), ((37, 21, 13), 8, 78), ((3, 2, 4), 8, 4)])
def test_balanced_segments_match_chunks(oracle_mod, n, TY, ncta):
    """The kernel's balanced split of the (column, node plane) units over ncta blocks,
    cut at column ends: segments cover every unit once, and the tiled apply over them is
    bit-identical to the z-chunked one (a segment recomputes the element layer below its
    first plane, so each node's sum order does not depend on the split)."""
    rng = np.random.default_rng(sum(n) + ncta)
    o = oracle_mod.Oracle(n, (1.1, 0.9, 0.7), E=3.0, nu=0.2, eta=1e-2)
    lam, mu = 3.0 * 0.2 / 1.2 / 0.6, 3.0 / 1.2 * 0.5
    v, x = rng.uniform(0, 1, o.N), rng.standard_normal(3 * o.N)
    mask, _ = o.bc(oracle_mod.rollers_face())
    bits = (mask.reshape(o.N, 3) * np.array([1, 2, 4])).sum(1).astype(np.uint8)
    h = tuple(L / (k - 1) for L, k in zip((1.1, 0.9, 0.7), n))
    ntx, nty = -(-(n[0] - 1) // 32), -(-(n[1] - 1) // TY)
    units = [(bx, by, z) for b in range(ncta) for bx, by, z0, z1 in km.segments(ntx, nty, n[2], ncta, b)
             for z in range(z0, z1)]
    assert sorted(units) == sorted((bx, by, z) for bx in range(ntx) for by in range(nty)
                                   for z in range(n[2]))
    ys = km.u_apply_tiled(x, v, bits, n, h, lam, mu, 1e-2, TY=TY, ncta=ncta)
    yc = km.u_apply_tiled(x, v, bits, n, h, lam, mu, 1e-2, TY=TY, zc=n[2])
    assert np.array_equal(ys, yc)


def test_modal_v_element_matches_gauss_sum(oracle_mod):
    """K_V,e x = sum_g [aeps w grad(phi_a).grad(x) + c_g phi_a x] from the element tables."""
    rng = np.random.default_rng(5)
    h = (0.3, 0.5, 0.7)
    w, phi, dphi = np.zeros(27), np.zeros(216), np.zeros(648)
    oracle_mod.lib().vfo_tables(*h, w, phi, dphi)
    phi, dphi = phi.reshape(8, 27), dphi.reshape(8, 3, 27)
    for _ in range(3):
        x, cg, aeps = rng.standard_normal(8), rng.uniform(0, 2, 27), rng.uniform(0.5, 2)
        K = np.einsum("g,adg,bdg->ab", w * aeps, dphi, dphi) + np.einsum("g,ag,bg->ab", cg, phi, phi)
        y = km.v_element(x, cg, aeps, h)
        assert np.abs(y - K @ x).max() <= 1e-13 * np.abs(K @ x).max()


@pytest.mark.parametrize("n,TY,ncta", [((37, 21, 13), 8, 7), ((70, 19, 11), 8, 5), ((37, 21, 13), 4, 3),
                                       ((37, 35, 9), 16, 4), ((3, 2, 4), 8, 3)])
def test_unit_lists_split_matches_plain(oracle_mod, n, TY, ncta):
    """The U apply split over unit lists (list 0: units whose adjacent element layers are
    constant-phase-field throughout the tile, on the fixed-weight kernel; list 1: the
    rest): the lists cover every (tile, plane) unit once, each block's list segments
    feed the fixed-weight operator only constant elements, and the two waves together
    give the plain balanced split's y bit for bit."""
    rng = np.random.default_rng(sum(n) + TY)
    o = oracle_mod.Oracle(n, (1.1, 0.9, 0.7), E=3.0, nu=0.2, eta=1e-2)
    lam, mu = 3.0 * 0.2 / 1.2 / 0.6, 3.0 / 1.2 * 0.5
    v = np.ones(o.N)
    vv = v.reshape(n[2], n[1], n[0])
    vv[n[2] // 2: n[2] // 2 + 2, : n[1] // 2, 3:] = rng.uniform(0, 1, vv[n[2] // 2: n[2] // 2 + 2, : n[1] // 2, 3:].shape)
    vv[:2] = 0.25
    x = rng.standard_normal(3 * o.N)
    mask, _ = o.bc(oracle_mod.rollers_face())
    bits = (mask.reshape(o.N, 3) * np.array([1, 2, 4])).sum(1).astype(np.uint8)
    h = tuple(L / (k - 1) for L, k in zip((1.1, 0.9, 0.7), n))
    ntx, nty = -(-(n[0] - 1) // 32), -(-(n[1] - 1) // TY)
    runs, start, tot = km.unit_lists(km.tile_layer_const(v, n, TY), n[2], ncta)
    segs = [[s for b in range(ncta) for s in km.list_segments(runs[l], start[l], tot[l], ncta, b, ntx)]
            for l in (0, 1)]
    units = sorted((bx, by, z) for l in (0, 1) for bx, by, z0, z1 in segs[l] for z in range(z0, z1))
    assert units == sorted((bx, by, z) for bx in range(ntx) for by in range(nty) for z in range(n[2]))
    assert tot[0] > 0 and tot[1] > 0

    def general(xn, vn):
        return km.u_element(xn, vn, lam, mu, 1e-2, h)

    def fixed_weight(xn, vn):
        assert (vn == vn[0]).all()
        return general(xn, vn)

    chunks = [s + (fixed_weight,) for s in segs[0]] + [s + (general,) for s in segs[1]]
    ys = km.u_apply_tiled(x, v, bits, n, h, lam, mu, 1e-2, TY=TY, chunks=chunks)
    yp = km.u_apply_tiled(x, v, bits, n, h, lam, mu, 1e-2, TY=TY, ncta=ncta)
    assert np.array_equal(ys, yp)
    assert np.abs(ys - o.u_apply(v, x, mask)).max() <= 1e-13 * np.abs(ys).max()
