"""GPU: the tensor-core element contraction (vfgpu_u_apply_tc: two GEMMs per tile of
128 elements on tcgen05.mma in split TF32, accumulators in tensor memory) against the
oracle's FP64 apply and the CUDA-core FP32 apply."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,l", [((17, 17, 17), (4.0, 4.0, 4.0)),
                                 ((37, 21, 13), (1.1, 0.9, 0.7)),
                                 ((66, 40, 35), (2.0, 1.3, 1.1))])
def test_tc_apply_matches_oracle(cuda, oracle_mod, n, l):
    import vpfhf_b200 as vg
    torch = cuda
    rng = np.random.default_rng(sum(n))
    E, nu, eta = 1e10, 0.25, 1e-8
    o = oracle_mod.Oracle(n, l, E=E, nu=nu, eta=eta)
    ctx = vg.VFContext(n, l, dict(E=E, nu=nu), eta=eta)
    ctx.set_bc(vg.rollers())
    mask, _ = o.bc(oracle_mod.rollers_face())
    # FP32-representable inputs, so that the oracle sees the values the kernel sees
    v = rng.uniform(0, 1, o.N).astype(np.float32).astype(np.float64)
    v[rng.uniform(size=o.N) < 0.1] = 0.0
    x = (rng.standard_normal(3 * o.N) * 1e-3).astype(np.float32).astype(np.float64)
    ctx.set_field("V", v)
    yref = o.u_apply(v, x, mask)
    xd = torch.from_numpy(x.astype(np.float32)).cuda()
    yd = torch.full_like(xd, float("nan"))
    ctx.u_apply_tc(xd, yd)
    torch.cuda.synchronize()
    assert not ctx.tc_error()
    y = yd.cpu().numpy().astype(np.float64)
    assert np.isfinite(y).all()
    err = np.linalg.norm(y - yref) / np.linalg.norm(yref)
    assert err <= 2e-6, err
    # against the CUDA-core FP32 apply of the same inputs
    y32 = ctx.u_apply(x, vg.MIXED)
    assert np.linalg.norm(y - y32) <= 4e-6 * np.linalg.norm(yref)
    ctx.close()
