"""Host-side logic of vpfhf_b200 (no GPU): crack construction, BC vector, options."""
import numpy as np
import pytest


@pytest.mark.parametrize("atnum,theta,phi,thick", [(1, 0, 0, 0.0), (2, 30, 45, 0.1),
                                                   (1, 120, 150, 0.05)])
def test_penny_crack_matches_oracle(oracle_mod, atnum, theta, phi, thick):
    import vpfhf_b200 as vg
    n, l = (17, 13, 21), (4.0, 3.0, 5.0)
    o = oracle_mod.Oracle(n, l, epsilon=0.3, atnum=atnum)
    ref = o.penny_v((2.0, 1.4, 2.6), 0.7, theta, phi, thick)
    got = vg.penny_crack_v(n, l, (2.0, 1.4, 2.6), 0.7, theta, phi, thick, epsilon=0.3, atnum=atnum)
    assert np.abs(got - ref).max() <= 1e-12


def test_bc_vector_matches_oracle(oracle_mod):
    """VecSetFromBC values for FIXED faces equal the oracle's Dirichlet values."""
    import vpfhf_b200 as vg
    n = (6, 5, 4)
    bcs = [vg.BCSpec(X0=(vg.BC_FIXED, -1.5), X1=(vg.BC_FIXED, 2.0), Z0=vg.BC_ZERO),
           vg.BCSpec(Y0=vg.BC_ONE, X1Y1Z1=(vg.BC_FIXED, 7.0)),
           vg.BCSpec(Z1=(vg.BC_FIXED, 3.0))]
    bcu = vg.bc_vector(n, bcs)
    o = oracle_mod.Oracle(n, (1, 1, 1))
    face = np.array([b.face for b in bcs], np.int32)
    vert = np.array([b.vertex for b in bcs], np.int32)
    mask, value = o.bc(face, vert, dof=3, bcu=bcu)
    assert np.array_equal(value[mask == 1], bcu[mask == 1])
    assert np.all(bcu[mask == 0] == 0)


def test_solve_opts_defaults():
    import vpfhf_b200 as vg
    o = vg.solve_opts(precision="mixed", ksp_maxit=77)
    assert o.precision == vg.MIXED and o.ksp_maxit == 77
    assert o.ksp_rtol == 1e-8 and o.ksp_atol == 1e-10 and o.snes_rtol == 1e-8
