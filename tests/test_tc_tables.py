"""CPU check of the tensor-core apply's two constant matrices (vfgpu_tc_tables, host
code of the library): the GEMM form GEMM1 -> pointwise degradation -> GEMM2, in FP64,
equals the reference's 27-point element matrix (VF_BilinearFormU3D_local,
VFMech.c:227-290) times the element's displacements."""
import ctypes as C

import numpy as np
import pytest


@pytest.mark.parametrize("h", [(0.3, 0.5, 0.7), (0.25, 0.25, 0.25)])
def test_tc_gemm_form_matches_element_matrix(oracle_mod, h):
    from vpfhf_b200 import _abi
    L = _abi.lib()
    B1 = np.zeros((32, 224))
    B2 = np.zeros((192, 32))
    assert L.vfgpu_tc_tables(*h, B1.ctypes.data_as(C.c_void_p), B2.ctypes.data_as(C.c_void_p)) == 0
    assert not B1[:, 216:].any() and not B2[:, 24:].any()
    assert not B2[63::64].any()  # the zero pad row of each pass
    E, nu, eta = 2.0, 0.3, 1e-3
    lam, mu = E * nu / (1 + nu) / (1 - 2 * nu), E / (1 + nu) / 2
    o = oracle_mod.Oracle((2, 2, 2), h, E=E, nu=nu, eta=eta)
    rng = np.random.default_rng(9)
    for _ in range(4):
        v, x = rng.uniform(0, 1, 8), rng.standard_normal(24)
        D1 = np.concatenate([x, v]) @ B1
        A2 = np.zeros(192)
        for g in range(27):
            T, Eq, V = D1[8 * g], D1[8 * g + 1:8 * g + 7], D1[8 * g + 7]
            s = V * V + eta
            k = 64 * (g // 9) + 7 * (g % 9)
            A2[k] = lam * s * T
            A2[k + 1:k + 7] = mu * s * Eq
        y = (A2 @ B2)[:24]
        yref = o.u_element_matrix(0, 0, 0, v) @ x
        assert np.abs(y - yref).max() <= 1e-13 * np.abs(yref).max()
