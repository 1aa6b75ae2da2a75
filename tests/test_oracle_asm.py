"""The assembled-method solves of the oracle (the timed CPU AM-step baseline: residuals
from re-formed element matrices, the Jacobian assembled into CSR every Newton iteration,
CG on the assembled matrix, VFMech.c:1555-1596, 1897-2029, 2772-2848, 2948-3027) give
the matrix-free oracle's solutions and iteration counts."""
import numpy as np
import pytest


@pytest.mark.parametrize("atnum", [1, 2])
def test_assembled_solves_match_matrix_free(oracle_mod, atnum):
    n, L = (13, 11, 9), 4.0
    h = max(L / (m - 1) for m in n)
    o = oracle_mod.Oracle(n, (L, L, L), E=1e10, nu=0.25, Gc=100.0, epsilon=2 * h, eta=1e-8,
                          atnum=atnum, pressurize=True, nthreads=2)
    V = o.penny_v((2.0, 2.0, 2.0), 0.9)
    p = np.full(o.N, 1e6)
    umask, uval = o.bc(oracle_mod.rollers_face())
    U1, U2 = np.zeros(3 * o.N), np.zeros(3 * o.N)
    s1 = o.step_u(U1, V, p=p, mask=umask, value=uval)
    s2, t_asm = o.step_u_asm(U2, V, p=p, mask=umask, value=uval)
    assert (s1.ksp_its, s1.newton_its) == (s2.ksp_its, s2.newton_its)
    assert np.abs(U1 - U2).max() <= 1e-12 * np.abs(U1).max()
    assert t_asm > 0
    lb = np.zeros(o.N)
    ub = V.copy() if atnum == 1 else np.ones(o.N)
    virrev = V if atnum == 2 else None
    V1, V2 = V.copy(), V.copy()
    t1 = o.step_v(V1, U1, lb, ub, p=p, virrev=virrev)
    t2, _ = o.step_v_asm(V2, U1, lb, ub, p=p, virrev=virrev)
    assert (t1.ksp_its, t1.newton_its, t1.reason) == (t2.ksp_its, t2.newton_its, t2.reason)
    assert np.abs(V1 - V2).max() <= 1e-12
