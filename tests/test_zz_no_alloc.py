"""vfgpu_u_apply_noalloc: the U apply for callers that cannot allocate device memory
while they run (it keeps its seam scratch in a fixed array inside the library).

Checked through the C ABI against the ctx-based vfgpu_u_apply and against the oracle's
matrix-free apply on two calls in a row (the second call reuses the scratch the first
one left behind).  This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(oracle_mod, o):
    mask, _ = o.bc(oracle_mod.rollers_face())
    return (mask.reshape(o.N, 3) * np.array([1, 2, 4])).sum(1).astype(np.uint8)


@pytest.mark.parametrize("n,l", [((37, 21, 13), (1.1, 0.9, 0.7)), ((65, 65, 65), (4.0, 4.0, 4.0)),
                                 ((129, 129, 129), (4.0, 4.0, 4.0))])
def test_noalloc_matches_ctx_apply_twice(cuda, oracle_mod, n, l):
    import vpfhf_b200 as vg
    from vpfhf_b200 import _abi
    torch = cuda
    E, nu, eta = 1e10, 0.25, 1e-8
    o = oracle_mod.Oracle(n, l)
    rng = np.random.default_rng(11)
    v = rng.uniform(0, 1, o.N)
    ctx = vg.VFContext(n, l, dict(E=E, nu=nu), eta=eta)
    ctx.set_bc(vg.rollers())
    ctx.set_field("V", v)
    grid = _abi.Grid(*n, *l)
    mp = _abi.MatProp(E, nu, 0.0, 0.0, 1.0)
    vd = torch.from_numpy(v).cuda()
    bits = torch.from_numpy(_bits(oracle_mod, o)).cuda()
    L = _abi.lib()
    for call in range(2):
        x = rng.standard_normal(3 * o.N) * 1e-4
        ref = ctx.u_apply(x, vg.FP64)
        xd = torch.from_numpy(x).cuda()
        yd = torch.full_like(xd, float("nan"))
        torch.cuda.synchronize()
        rc = L.vfgpu_u_apply_noalloc(C.byref(grid), C.byref(mp), eta, vd.data_ptr(),
                                     bits.data_ptr(), xd.data_ptr(), yd.data_ptr(), None)
        assert rc == 0, L.vfgpu_last_error().decode()
        torch.cuda.synchronize()
        y = yd.cpu().numpy()
        assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max(), call
        if o.N <= 65 ** 3:  # the oracle's apply (Dirichlet rows y = x) at the same tolerance
            mask, _ = o.bc(oracle_mod.rollers_face())
            yo = oracle_mod.Oracle(n, l, E=E, nu=nu, eta=eta).u_apply(v, x, mask)
            assert np.abs(y - yo).max() <= 1e-12 * np.abs(yo).max(), call
    ctx.close()


def test_noalloc_rejects_overlapping_x_and_y(cuda):
    """The apply is out of place: x and y that share memory are refused before any launch."""
    from vpfhf_b200 import _abi
    torch = cuda
    n = (9, 9, 9)
    grid = _abi.Grid(*n, 1.0, 1.0, 1.0)
    mp = _abi.MatProp(1e10, 0.25, 0.0, 0.0, 1.0)
    N = 9 ** 3
    v = torch.ones(N, dtype=torch.float64, device="cuda")
    buf = torch.zeros(3 * N + 8, dtype=torch.float64, device="cuda")
    L = _abi.lib()
    for off in (0, 8):  # the same array, and an array shifted by 8 doubles
        rc = L.vfgpu_u_apply_noalloc(C.byref(grid), C.byref(mp), 1e-8, v.data_ptr(), None,
                                     buf.data_ptr(), buf.data_ptr() + off * 8, None)
        assert rc == _abi.ERR_INVALID
        assert "overlap" in L.vfgpu_last_error().decode()


def test_noalloc_rejects_grids_beyond_the_fixed_scratch(cuda):
    from vpfhf_b200 import _abi
    torch = cuda
    n = (161, 161, 161)
    grid = _abi.Grid(*n, 4.0, 4.0, 4.0)
    mp = _abi.MatProp(1e10, 0.25, 0.0, 0.0, 1.0)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")  # never dereferenced: size check first
    L = _abi.lib()
    rc = L.vfgpu_u_apply_noalloc(C.byref(grid), C.byref(mp), 1e-8, d.data_ptr(), None,
                                 d.data_ptr(), d.data_ptr(), None)
    assert rc == _abi.ERR_INVALID
    assert "scratch" in L.vfgpu_last_error().decode()
