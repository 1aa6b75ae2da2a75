"""The oracle's restatement of the flow-coupling boundary (VFPermfield.c): fracture width
(UpdateFractureWidth, :267-562), cell-to-node average (CellToNodeInterpolation,
:1156-1330), well rate (VolumetricFractureWellRate, :1513-1604) and the integration
length (VFCommon.c:897-914), against answers worked out by hand.

The reference's width code needs PETSc (DMDA ghost arrays, coordinates) and is not
compiled here, so these known answers pin the restatement:
- V linear in z with slope b and U constant c e_z: grad V . U = b c everywhere, every
  march step adds b c len / 2 (the segment rule integrates and halves), and with
  L / len = 166.4 both marches take 165 steps: width = 165 b c len, len = hz / 20;
- the integrated grad V is 165 b len, so pmult = 0 once that exceeds width_tol;
- U -> 2U doubles every width bit for bit; V = 1 gives no band; V = 1/2 everywhere
  stalls every cell (zero gradient: the reference's march would not end);
- a constant cell field interpolates to the same constant; an interior node is the
  mean of its 8 cells; the well rate of V linear in z and a constant rate r is
  r b |box|."""
import numpy as np
import pytest


def _linear_case(oracle_mod, b_h=0.03, c=1e-3):
    n, L = (9, 9, 25), (1.0, 1.0, 3.0)
    h = L[2] / (n[2] - 1)
    o = oracle_mod.Oracle(n, L, E=1.0, nu=0.3, Gc=1.0, epsilon=1.33 * h, eta=1e-8, atnum=1)
    z = np.repeat(np.arange(n[2]) * h, n[0] * n[1])
    b = b_h / h
    v = 0.5 + b * (z - 1.5)
    u = np.zeros(3 * o.N)
    u[2::3] = c
    return o, u, v, b, c, h


def test_width_linear_v_known_answer(oracle_mod):
    o, u, v, b, c, h = _linear_case(oracle_mod)
    wc, wn, pm, st = o.fracture_width(u, v, int_length=8.32 * h, width_tol=0.1)
    assert st == 0
    expect = 165 * b * c * (h / 20)
    assert np.allclose(wc, expect, rtol=1e-12, atol=0)
    assert np.allclose(wn, expect, rtol=1e-12, atol=0)
    assert (pm == 0).all()  # 165 b len = 0.2475 > 0.1
    # a tolerance above the integrated gradient keeps the permeability multiplier 1
    _, _, pm2, _ = o.fracture_width(u, v, int_length=8.32 * h, width_tol=0.3)
    assert (pm2 == 1).all()
    # removeTipEffect zeroes the width where the integrated gradient exceeds width_tol
    wc3, _, _, _ = o.fracture_width(u, v, int_length=8.32 * h, width_tol=0.1, remove_tip=True)
    assert (wc3 == 0).all()


def test_width_properties(oracle_mod):
    n, L = 17, 4.0
    h = L / (n - 1)
    o = oracle_mod.Oracle((n, n, n), (L, L, L), E=1e10, nu=0.25, Gc=100.0, epsilon=2 * h,
                          eta=1e-8, atnum=1, pressurize=True)
    v = o.penny_v((2.0, 2.0, 2.0), 0.8)
    z = np.repeat(np.arange(n) * h, n * n)
    u = np.zeros(3 * o.N)
    u[2::3] = np.where(z > 2.0, 0.5e-3, -0.5e-3)
    wc, wn, pm, st = o.fracture_width(u, v)
    assert st == 0 and wc.max() > 0 and (wc >= 0).all()
    assert set(np.unique(pm)) <= {0.0, 1.0}
    wc2, _, pm2, _ = o.fracture_width(2 * u, v)
    assert np.array_equal(wc2, 2 * wc) and np.array_equal(pm2, pm)
    # mirror symmetry of the set-up in x: the width field is mirrored (a march may end
    # one step apart on the two sides when lc meets the integration length in rounding)
    W = wc.reshape(n - 1, n - 1, n - 1)
    close = np.isclose(W, W[:, :, ::-1], rtol=1e-9, atol=1e-15)
    assert close.mean() > 0.99 and np.allclose(W, W[:, :, ::-1], rtol=1e-3, atol=1e-15)
    # no band without a crack
    wc0, _, pm0, st0 = o.fracture_width(u, np.ones(o.N))
    assert (wc0 == 0).all() and (pm0 == 1).all() and st0 == 0
    # zero gradient inside the band: every cell stalls and keeps width 0
    wcs, _, _, sts = o.fracture_width(u, np.full(o.N, 0.5))
    assert sts == (n - 1) ** 3 and (wcs == 0).all()


def test_width_int_length(oracle_mod):
    h = 4.0 / 16
    o = oracle_mod.Oracle((17, 17, 17), (4.0, 4.0, 4.0), E=1.0, nu=0.3, Gc=1.0, epsilon=2 * h)
    assert o.width_int_length() == pytest.approx(3 * h + 8 * h, rel=1e-15)
    # the reference's comparison chain: bx == by < bz picks bz
    o2 = oracle_mod.Oracle((17, 17, 9), (4.0, 4.0, 4.0), E=1.0, nu=0.3, Gc=1.0, epsilon=0.1)
    assert o2.width_int_length() == pytest.approx(3 * 0.5 + 0.4, rel=1e-15)
    o3 = oracle_mod.Oracle((9, 17, 17), (4.0, 4.0, 4.0), E=1.0, nu=0.3, Gc=1.0, epsilon=0.1)
    assert o3.width_int_length() == pytest.approx(3 * 0.25 + 0.4, rel=1e-15)


def test_cell_to_node_and_well_rate(oracle_mod):
    n, L = (6, 5, 7), (1.0, 2.0, 3.0)
    o = oracle_mod.Oracle(n, L, E=1.0, nu=0.3, Gc=1.0, epsilon=0.1)
    nc = 5 * 4 * 6
    assert np.allclose(o.cell_to_node(np.full(nc, 2.5)), 2.5, rtol=1e-15)
    rng = np.random.default_rng(3)
    cell = rng.standard_normal(nc)
    nodev = o.cell_to_node(cell)
    C = cell.reshape(6, 4, 5)
    i, j, k = 2, 1, 3
    assert nodev[(k * n[1] + j) * n[0] + i] == pytest.approx(C[k - 1:k + 1, j - 1:j + 1, i - 1:i + 1].mean(), rel=1e-14)
    # corner node: its one cell
    assert nodev[0] == pytest.approx(C[0, 0, 0], rel=1e-14)
    z = np.repeat(np.arange(n[2]) * (L[2] / (n[2] - 1)), n[0] * n[1])
    b = 0.2
    rate = o.fracture_well_rate(0.1 + b * z, np.full(o.N, 3.0))
    assert rate == pytest.approx(3.0 * b * L[0] * L[1] * L[2], rel=1e-12)
