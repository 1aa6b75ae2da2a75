"""UNILATERAL_NOCOMPRESSION in the oracle (VFMech.c:115-218, 299-376, 456-524, 819-908,
2125-2153): the matrix-free form against the assembled element matrices, the
tensile limit equal to the plain model, and a Newton solve that converges."""
import numpy as np
import pytest

N3 = (7, 6, 5)
L3 = (1.2, 1.0, 0.8)


def _problem(oracle_mod, unilateral, alpha=0.0, beta=0.0):
    return oracle_mod.Oracle(N3, L3, E=3.0, nu=0.27, Gc=1.0, alpha=alpha, beta=beta, eta=1e-3,
                             epsilon=0.3, unilateral=unilateral, pressurize=True)


def _grid():
    xs = [np.arange(k) * (l / (k - 1)) for k, l in zip(N3, L3)]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    return X.ravel(), Y.ravel(), Z.ravel()


def test_matrix_free_matches_element_matrices(oracle_mod):
    rng = np.random.default_rng(0)
    o = _problem(oracle_mod, 1)
    v = rng.uniform(0, 1, o.N)
    u0 = rng.standard_normal(3 * o.N)  # both signs of tr(eps) occur
    x = rng.standard_normal(3 * o.N)
    y = o.u_apply_u(u0, v, x)
    yr = o.u_apply_u(u0, v, x, ref=True)
    assert np.abs(y - yr).max() <= 1e-13 * np.abs(yr).max()
    # the sign pattern matters: not the plain operator
    assert np.abs(y - o.u_apply(v, x)).max() > 1e-6 * np.abs(yr).max()


def test_tensile_limit_is_the_plain_model(oracle_mod):
    """With tr(eps(u0)) > 0 everywhere the NOCOMPRESSION forms are the plain ones."""
    rng = np.random.default_rng(1)
    X, Y, Z = _grid()
    u0 = np.stack([0.3 * X, 0.2 * Y, 0.1 * Z], -1).ravel()
    v = rng.uniform(0, 1, X.size)
    x = rng.standard_normal(3 * X.size)
    theta, p = rng.uniform(0, 5, X.size), rng.uniform(0, 2, X.size)
    onc = _problem(oracle_mod, 1, alpha=1e-2, beta=0.6)
    o = _problem(oracle_mod, 0, alpha=1e-2, beta=0.6)
    y, y0 = onc.u_apply_u(u0, v, x), o.u_apply(v, x)
    assert np.abs(y - y0).max() <= 1e-13 * np.abs(y0).max()
    f, f0 = onc.u_rhs_u(u0, v, theta, None, p), o.u_rhs(v, theta, None, p)
    assert np.abs(f - f0).max() <= 1e-13 * np.abs(f0).max()
    # V coupling with theta = 0: W_S + W_D = W
    xv = rng.standard_normal(X.size)
    assert np.allclose(onc.v_apply(u0, xv), o.v_apply(u0, xv), rtol=0, atol=1e-12)


def test_compression_keeps_the_spherical_stiffness(oracle_mod):
    rng = np.random.default_rng(2)
    X, Y, Z = _grid()
    u0 = np.stack([-0.3 * X, -0.2 * Y, -0.1 * Z], -1).ravel()  # tr(eps) < 0 everywhere
    v = rng.uniform(0, 1, X.size)
    onc, o = _problem(oracle_mod, 1), _problem(oracle_mod, 0)
    for _ in range(3):
        x = rng.standard_normal(3 * X.size)
        assert x @ onc.u_apply_u(u0, v, x) >= x @ o.u_apply(v, x)
    e_nc, _ = onc.u_energy(u0, v)
    e0, _ = o.u_energy(u0, v)
    assert e_nc > e0


def test_residual_is_operator_at_u_minus_load(oracle_mod):
    rng = np.random.default_rng(3)
    o = _problem(oracle_mod, 1, alpha=1e-2, beta=0.6)
    v = rng.uniform(0, 1, o.N)
    u = rng.standard_normal(3 * o.N) * 0.1
    theta, p = rng.uniform(0, 5, o.N), rng.uniform(0, 2, o.N)
    F = o.u_residual_ref(u, v, theta, None, p)
    Fm = o.u_apply_u(u, v, u) - o.u_rhs_u(u, v, theta, None, p)
    assert np.abs(F - Fm).max() <= 1e-12 * np.abs(F).max()


def test_newton_converges_under_compression(oracle_mod):
    """A cracked block squeezed across the crack (Z1 pushed down, rollers elsewhere):
    Newton with the re-formed NOCOMPRESSION Jacobian converges, and the crack does
    not close as freely as in the plain model."""
    n, L = (9, 9, 9), (1.0, 1.0, 1.0)
    res = {}
    for uni in (0, 1):
        o = oracle_mod.Oracle(n, L, E=1.0, nu=0.3, Gc=1.0, eta=1e-6, epsilon=0.25,
                              unilateral=uni, pressurize=False)
        v = o.penny_v((0.5, 0.5, 0.5), 2.0, thickness=0.15)  # a broken layer across the block
        face = np.zeros((3, 6), np.int32)
        face[0, :2] = face[1, 2:4] = oracle_mod.ZERO
        face[2, 4] = oracle_mod.ZERO
        face[2, 5] = oracle_mod.FIXED
        bcu = np.zeros(3 * o.N)
        bcu[2::3] = -0.01
        mask, val = o.bc(face, bcu=bcu)
        u = np.zeros(3 * o.N)
        u[mask == 1] = val[mask == 1]
        st = o.step_u(u, v, mask=mask, value=val)
        assert st.reason > 0, st.reason
        F = o.u_residual_ref(u, v, mask=mask, value=val)
        assert np.abs(F).max() <= 1e-6 * max(st.fnorm0, 1e-30) + 1e-12
        res[uni] = (o.u_energy(u, v)[0], st.newton_its)
    assert res[1][0] > 10 * res[0][0]  # the squeezed crack stores volumetric energy
