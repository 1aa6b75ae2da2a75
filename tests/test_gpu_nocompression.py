"""GPU: UNILATERAL_NOCOMPRESSION against the oracle -- operator linearised at the
resident U, U and V residuals, energies, and StepU's Newton solve of a crack
squeezed across its faces."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(oracle_mod, n=(17, 13, 11), L=(2.0, 1.5, 1.2), alpha=1e-5, beta=0.7, atnum=1):
    import vpfhf_b200 as vg
    kw = dict(E=1e10, nu=0.25, Gc=100.0, epsilon=0.3, eta=1e-8, atnum=atnum)
    o = oracle_mod.Oracle(n, L, alpha=alpha, beta=beta, pressurize=True, unilateral=1, **kw)
    ctx = vg.VFContext(n, L, dict(E=kw["E"], nu=kw["nu"], Gc=kw["Gc"], alpha=alpha, beta=beta),
                       epsilon=kw["epsilon"], eta=kw["eta"], atnum=atnum, pressurize=True)
    ctx.set_unilateral("nocompression")
    v = o.penny_v((1.0, 0.75, 0.6), 0.5, thickness=0.1)
    ctx.set_field("V", v)
    ctx.set_field("VIrrev", v)
    return o, ctx, v


def test_operator_and_residuals(cuda, oracle_mod):
    import vpfhf_b200 as vg
    rng = np.random.default_rng(11)
    o, ctx, v = _pair(oracle_mod)
    u = rng.standard_normal(3 * o.N) * 1e-4  # tr(eps) of both signs
    theta, p = rng.uniform(0, 10, o.N), rng.uniform(0, 2e6, o.N)
    ctx.set_field("U", u)
    ctx.set_field("theta", theta)
    ctx.set_field("pressure", p)
    x = rng.standard_normal(3 * o.N)
    y = ctx.u_apply(x, vg.FP64)
    yr = o.u_apply_u(u, v, x)
    assert np.abs(y - yr).max() <= 1e-12 * np.abs(yr).max()
    y32 = ctx.u_apply(x, vg.MIXED)
    assert np.linalg.norm(y32 - yr) <= 2e-6 * np.linalg.norm(yr)
    F = ctx.u_residual()
    Fr = o.u_residual_ref(u, v, theta, None, p)
    assert np.abs(F - Fr).max() <= 1e-11 * np.abs(Fr).max()
    Fv = ctx.v_residual()
    Fvr = o.v_residual_ref(u, v, theta, None, p, v)
    assert np.abs(Fv - Fvr).max() <= 1e-11 * np.abs(Fvr).max()
    el, _, pw = ctx.u_energy()
    el_o, pw_o = o.u_energy(u, v, theta, None, p)
    assert el == pytest.approx(el_o, rel=1e-12) and pw == pytest.approx(pw_o, rel=1e-12)
    ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_squeezed_crack_newton(cuda, oracle_mod, precision):
    """A broken layer pushed shut (Z1 displaced down, rollers elsewhere): the
    NOCOMPRESSION Newton iterations converge to the oracle's solution."""
    import vpfhf_b200 as vg
    n, L = (13, 13, 13), (1.0, 1.0, 1.0)
    o = oracle_mod.Oracle(n, L, E=1.0, nu=0.3, Gc=1.0, eta=1e-6, epsilon=0.25, unilateral=1,
                          pressurize=False)
    ctx = vg.VFContext(n, L, dict(E=1.0, nu=0.3, Gc=1.0), epsilon=0.25, eta=1e-6, atnum=1)
    ctx.set_unilateral(1)
    v = o.penny_v((0.5, 0.5, 0.5), 2.0, thickness=0.15)
    ctx.set_field("V", v)
    face = np.zeros((3, 6), np.int32)
    face[0, :2] = face[1, 2:4] = oracle_mod.ZERO
    face[2, 4] = oracle_mod.ZERO
    face[2, 5] = oracle_mod.FIXED
    bcu = np.zeros(3 * o.N)
    bcu[2::3] = -0.01
    mask, val = o.bc(face, bcu=bcu)
    uo = np.zeros(3 * o.N)
    uo[mask == 1] = val[mask == 1]
    st = o.step_u(uo, v, mask=mask, value=val)
    assert st.reason > 0
    bc = [vg.BCSpec(X0=vg.BC_ZERO, X1=vg.BC_ZERO), vg.BCSpec(Y0=vg.BC_ZERO, Y1=vg.BC_ZERO),
          vg.BCSpec(Z0=vg.BC_ZERO, Z1=(vg.BC_FIXED, -0.01))]
    ctx.set_bc(bc)
    ctx.set_field("BCU", bcu)
    ctx.time_step_prepare()
    rc, s = ctx.step_u(dict(precision=precision))
    assert rc == 0 and s["reason"] > 0, s
    assert s["newton_its"] >= 2  # the sign pattern changes after the first step
    ug = ctx.get_field("U")
    assert np.linalg.norm(ug - uo) <= 1e-6 * np.linalg.norm(uo)
    el, _, _ = ctx.u_energy()
    assert el == pytest.approx(o.u_energy(uo, v)[0], rel=1e-6)
    ctx.close()
