"""GPU: the flow-coupling boundary (width.cu) against the oracle -- fracture width per
cell and node, the permeability multiplier and the stalled-march count bit for bit
(same operation order, no FMA contraction), the well rate to 1e-12."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx(vg, n, L, eps):
    ctx = vg.VFContext(n, L, dict(E=1e10, nu=0.25, Gc=100.0), epsilon=eps, eta=1e-8, atnum=1,
                       pressurize=True)
    ctx.set_bc(vg.rollers())
    return ctx


@pytest.mark.parametrize("case", ["solved", "inclined_random_u"])
def test_width_matches_oracle(cuda, oracle_mod, case):
    import vpfhf_b200 as vg
    n, L = (33, 33, 33), (4.0, 4.0, 4.0)
    h = L[0] / (n[0] - 1)
    o = oracle_mod.Oracle(n, L, E=1e10, nu=0.25, Gc=100.0, epsilon=2 * h, eta=1e-8, atnum=1,
                          pressurize=True)
    ctx = _ctx(vg, n, L, 2 * h)
    if case == "solved":
        ctx.set_field("pressure", np.full(ctx.N, 1e6))
        ctx.init_cracks([dict(center=(2.0, 2.0, 2.0), r=0.9, theta=0.0, phi=0.0, thickness=2 * h)])
        ctx.time_step_prepare()
        rc, st = ctx.step_u()
        assert rc == 0, st
        u, v = ctx.get_field("U"), ctx.get_field("V")
    else:
        v = o.penny_v((1.9, 2.1, 2.0), 1.0, theta=35.0, phi=50.0)
        u = np.random.default_rng(8).standard_normal(3 * o.N) * 1e-4
        ctx.set_field("V", v)
        ctx.set_field("U", u)
    wc, wn, pm, st = ctx.update_fracture_width()
    wco, wno, pmo, sto = o.fracture_width(u, v)
    assert (wc > 0).sum() > 100
    assert np.array_equal(wc, wco) and np.array_equal(pm, pmo) and st == sto
    assert np.array_equal(wn, wno)
    # options: an explicit integration length, a tolerance, removeTipEffect
    wc2, _, pm2, _ = ctx.update_fracture_width(int_length=5 * h, width_tol=0.05,
                                               remove_tip_effect=True)
    wco2, _, pmo2, _ = o.fracture_width(u, v, int_length=5 * h, width_tol=0.05, remove_tip=True)
    assert np.array_equal(wc2, wco2) and np.array_equal(pm2, pmo2)
    ctx.close()


def test_width_known_answer_and_stall(cuda, oracle_mod):
    import vpfhf_b200 as vg
    n, L = (9, 9, 25), (1.0, 1.0, 3.0)
    h = L[2] / (n[2] - 1)
    ctx = _ctx(vg, n, L, 1.33 * h)
    z = np.repeat(np.arange(n[2]) * h, n[0] * n[1])
    b, c = 0.03 / h, 1e-3
    u = np.zeros(3 * ctx.N)
    u[2::3] = c
    ctx.set_field("U", u)
    ctx.set_field("V", 0.5 + b * (z - 1.5))
    wc, wn, pm, st = ctx.update_fracture_width(int_length=8.32 * h)
    assert st == 0 and np.allclose(wc, 165 * b * c * h / 20, rtol=1e-12, atol=0)
    assert np.allclose(wn, 165 * b * c * h / 20, rtol=1e-12, atol=0) and (pm == 0).all()
    ctx.set_field("V", np.full(ctx.N, 0.5))
    wc, _, _, st = ctx.update_fracture_width()
    assert st == 8 * 8 * 24 and (wc == 0).all()
    ctx.close()


def test_well_rate_matches_oracle(cuda, oracle_mod):
    import vpfhf_b200 as vg
    n, L = (33, 25, 17), (4.0, 3.0, 2.0)
    o = oracle_mod.Oracle(n, L, E=1e10, nu=0.25, Gc=100.0, epsilon=0.25, eta=1e-8, atnum=2)
    ctx = _ctx(vg, n, L, 0.25)
    v = o.penny_v((2.0, 1.5, 1.0), 0.7, theta=20.0, phi=10.0)
    reg = np.random.default_rng(4).uniform(0, 2, o.N)
    ctx.set_field("V", v)
    r = ctx.fracture_well_rate(reg)
    assert r == pytest.approx(o.fracture_well_rate(v, reg), rel=1e-12)
    ctx.close()


def test_cell_to_node_and_cov_nodes_match_oracle(cuda, oracle_mod):
    """CellToNodeInterpolation on the device (gather over each node's cells in the
    reference's scatter order) is the oracle's to the bit; with the per-cell crack
    opening it gives VolumetricCrackOpening's fields->VolCrackOpening."""
    import vpfhf_b200 as vg
    n, L = (21, 17, 13), (2.0, 1.6, 1.2)
    o = oracle_mod.Oracle(n, L, E=1e10, nu=0.25, Gc=100.0, epsilon=0.2, eta=1e-8, atnum=1)
    ctx = _ctx(vg, n, L, 0.2)
    rng = np.random.default_rng(12)
    cell = rng.standard_normal(20 * 16 * 12)
    assert np.array_equal(ctx.cell_to_node(cell), o.cell_to_node(cell))
    v = o.penny_v((1.0, 0.8, 0.6), 0.5, theta=10.0, phi=30.0)
    u = rng.standard_normal(3 * o.N) * 1e-3
    ctx.set_field("V", v)
    ctx.set_field("U", u)
    cov, cellcov = ctx.crack_opening(cell=True)
    cov_o, cellcov_o = o.cov(u, v, cell=True)
    assert cov == pytest.approx(cov_o, rel=1e-12)
    assert np.allclose(ctx.cell_to_node(cellcov), o.cell_to_node(cellcov_o), rtol=1e-10, atol=1e-18)
    ctx.close()
