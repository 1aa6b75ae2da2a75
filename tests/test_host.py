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


def test_mg_hierarchy_levels():
    """The multigrid hierarchy: an axis with >= 9 nodes goes to n/2 + 1 nodes
    (ceil(cells / 2) cells), the others keep theirs, until no axis has 9 nodes."""
    import vpfhf_b200 as vg
    lv, nb = vg.mg_hierarchy((129, 129, 129))
    assert lv == [(129,) * 3, (65,) * 3, (33,) * 3, (17,) * 3, (9,) * 3, (5,) * 3] and nb > 0
    assert [d[0] for d in vg.mg_hierarchy((128, 128, 128))[0]] == [128, 65, 33, 17, 9, 5]
    assert [d[0] for d in vg.mg_hierarchy((48, 48, 48))[0]] == [48, 25, 13, 7]
    assert vg.mg_hierarchy((40, 33, 12))[0] == [(40, 33, 12), (21, 17, 7), (11, 9, 7), (6, 5, 7)]
    assert vg.mg_hierarchy((8, 8, 8))[0] == [(8, 8, 8)]  # refused by a pc="mg" solve
    # FP64 hierarchy holds more bytes than the FP32 one; the estimate grows with the grid
    n32 = vg.mg_hierarchy((65, 65, 65), precision=vg.MIXED)[1]
    n64 = vg.mg_hierarchy((65, 65, 65), precision=vg.FP64)[1]
    assert n64 > n32 > vg.mg_hierarchy((33, 33, 33))[1] > 0
    assert vg.mg_hierarchy((8, 8, 8))[1] == 0
