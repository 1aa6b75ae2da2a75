"""GPU parity of the matrix-free U operator (vfgpu_u_apply) against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRIDS = [((5, 5, 5), (1.0, 1.0, 1.0)),
         ((17, 17, 17), (4.0, 4.0, 4.0)),
         ((37, 21, 13), (1.1, 0.9, 0.7)),      # ragged tiles, x- and y-seams
         ((41, 41, 41), (4.0, 4.0, 4.0)),      # the 41^3 penny-crack grid
         ((66, 40, 35), (2.0, 1.3, 1.1))]


def _setup(oracle_mod, n, l, seed, cellE=False):
    import vpfhf_b200 as vg
    rng = np.random.default_rng(seed)
    E, nu, eta = 1e10, 0.25, 1e-8
    cE = None
    if cellE:
        cE = np.exp(np.log(E) + 0.5 * rng.standard_normal((n[0] - 1) * (n[1] - 1) * (n[2] - 1)))
        cE = cE.astype(np.float32).astype(np.float64)  # the device stores per-cell E in FP32
    o = oracle_mod.Oracle(n, l, E=E, nu=nu, eta=eta, cellE=cE)
    ctx = vg.VFContext(n, l, dict(E=E, nu=nu), eta=eta)
    if cE is not None:
        ctx.set_cell_modulus(cE)
    ctx.set_bc(vg.rollers())
    mask, _ = o.bc(oracle_mod.rollers_face())
    v = rng.uniform(0, 1, o.N)
    v[rng.uniform(size=o.N) < 0.1] = 0.0                 # cracked nodes: s = eta
    ctx.set_field("V", v)
    x = rng.standard_normal(3 * o.N) * 1e-3
    return o, ctx, v, x, mask


@pytest.mark.parametrize("n,l", GRIDS)
def test_u_apply_fp64(cuda, oracle_mod, n, l):
    import vpfhf_b200 as vg
    o, ctx, v, x, mask = _setup(oracle_mod, n, l, 1)
    yref = o.u_apply(v, x, mask)
    y = ctx.u_apply(x, vg.FP64)
    assert np.abs(y - yref).max() <= 1e-12 * np.abs(yref).max()
    # device pointers are used in place
    xd = cuda.from_numpy(x).cuda()
    yd = ctx.u_apply(xd, vg.FP64)
    assert np.array_equal(yd.cpu().numpy(), y)
    # deterministic: identical bits on a second call
    assert np.array_equal(ctx.u_apply(x, vg.FP64), y)
    ctx.close()


@pytest.mark.parametrize("n,l", GRIDS[1:4])
def test_u_apply_fp32(cuda, oracle_mod, n, l):
    import vpfhf_b200 as vg
    o, ctx, v, x, mask = _setup(oracle_mod, n, l, 2)
    yref = o.u_apply(v, x, mask)
    y = ctx.u_apply(x, vg.MIXED)
    # FP32 operator: normwise relative error at the FP32 level
    assert np.linalg.norm(y - yref) <= 2e-6 * np.linalg.norm(yref)
    ctx.close()


def test_u_apply_cell_modulus(cuda, oracle_mod):
    import vpfhf_b200 as vg
    o, ctx, v, x, mask = _setup(oracle_mod, (37, 21, 13), (1.1, 0.9, 0.7), 3, cellE=True)
    yref = o.u_apply(v, x, mask)
    y = ctx.u_apply(x, vg.FP64)
    assert np.abs(y - yref).max() <= 1e-12 * np.abs(yref).max()
    ctx.close()


@pytest.mark.parametrize("unilateral", [0, 1])
def test_u_apply_host_pipeline_matches_device(cuda, oracle_mod, unilateral):
    """Host buffers go through the slab pipeline (copies up, slab applies
    and copies down overlapping on three streams): bit-identical to the device-buffer
    apply, with a per-cell modulus, slabs of 5 planes (45 planes) and, under
    NOCOMPRESSION, the per-cell compression bits; pageable and pinned host memory."""
    import vpfhf_b200 as vg
    n, l = (23, 19, 45), (1.0, 0.8, 2.0)
    o, ctx, v, x, mask = _setup(oracle_mod, n, l, 7, cellE=True)
    if unilateral:
        ctx.set_unilateral(1)
        ctx.set_field("U", np.random.default_rng(3).standard_normal(3 * o.N) * 1e-4)
    y = ctx.u_apply(x, vg.FP64)
    yd = ctx.u_apply(cuda.from_numpy(x).cuda(), vg.FP64).cpu().numpy()
    assert np.array_equal(y, yd)
    if not unilateral:
        yref = o.u_apply(v, x, mask)
        assert np.abs(y - yref).max() <= 1e-12 * np.abs(yref).max()
    xp = cuda.empty(3 * o.N, dtype=cuda.float64, pin_memory=True)
    yp = cuda.empty(3 * o.N, dtype=cuda.float64, pin_memory=True)
    xp.numpy()[:] = x
    for _ in range(2):
        ctx.u_apply(xp.numpy(), vg.FP64, out=yp.numpy())
        assert np.array_equal(yp.numpy(), y)
    ctx.close()


@pytest.mark.parametrize("n,l,cellE,split", [((41, 41, 41), (4.0, 4.0, 4.0), False, "auto"),
                                             ((41, 41, 41), (4.0, 4.0, 4.0), True, "auto"),
                                             ((37, 21, 13), (1.1, 0.9, 0.7), False, "auto"),
                                             ((41, 41, 41), (4.0, 4.0, 4.0), True, "on"),
                                             ((37, 21, 13), (1.1, 0.9, 0.7), False, "on")])
def test_u_apply_constant_phase_field_elements(cuda, oracle_mod, n, l, cellE, split):
    """Mostly intact phase field (v = 1 away from a penny crack, a block of a constant
    v = 0.4 and a random block): elements whose 8 nodal v are equal take the
    fixed-weight element, the rest the row closed form; FP64 at 1e-12 and FP32 at
    2e-6 normwise against the oracle, on cubic and non-cubic cells, with per-cell
    modulus, in one wave and split by phase field."""
    import vpfhf_b200 as vg
    o, ctx, _, x, mask = _setup(oracle_mod, n, l, 5, cellE=cellE)
    ctx.set_u_split(split)
    rng = np.random.default_rng(6)
    pen = oracle_mod.Oracle(n, l, epsilon=2 * max(li / (ni - 1) for li, ni in zip(l, n)))
    v = pen.penny_v(tuple(li / 2 for li in l), 0.25 * min(l))
    vv = v.reshape(n[2], n[1], n[0])
    vv[:n[2] // 3, :n[1] // 3, :n[0] // 3] = 0.4
    vv[-n[2] // 4:, -n[1] // 4:, -n[0] // 4:] = rng.uniform(0, 1, vv[-n[2] // 4:, -n[1] // 4:, -n[0] // 4:].shape)
    v = vv.reshape(-1).copy()
    ctx.set_field("V", v)
    yref = o.u_apply(v, x, mask)
    y = ctx.u_apply(x, vg.FP64)
    assert np.abs(y - yref).max() <= 1e-12 * np.abs(yref).max()
    y32 = ctx.u_apply(x, vg.MIXED)
    assert np.linalg.norm(y32 - yref) <= 2e-6 * np.linalg.norm(yref)
    ctx.close()


@pytest.mark.parametrize("n,l", [((66, 40, 35), (2.0, 1.3, 1.1)), ((23, 19, 45), (1.0, 0.8, 2.0))])
def test_unit_lists_split(cuda, oracle_mod, n, l):
    """U applies split by phase field (vfgpu_set_u_split on: the (tile, plane) units over
    the fixed-weight kernel and the general one, unit lists rebuilt when v changes):
    bit-identical to one wave (split off, FP64 and FP32), to vfgpu_u_apply_noalloc and to
    the host slab pipeline (sub-grids, one wave), following each change of v (intact field
    with a cracked blob, random, intact, blob again); FP32 at 2e-6 against the oracle."""
    import ctypes as C

    import vpfhf_b200 as vg
    from vpfhf_b200 import _abi
    torch = cuda
    E, nu, eta = 1e10, 0.25, 1e-8
    o, ctx, _, x, mask = _setup(oracle_mod, n, l, 9)
    rng = np.random.default_rng(10)
    blob = np.ones(o.N)
    bb = blob.reshape(n[2], n[1], n[0])
    bb[n[2] // 3: n[2] // 2, n[1] // 4: n[1] // 2, 5: 40] = rng.uniform(0, 1, bb[n[2] // 3: n[2] // 2, n[1] // 4: n[1] // 2, 5: 40].shape)
    bb[-4:, :9, :] = 0.3
    bits = torch.from_numpy((mask.reshape(o.N, 3) * np.array([1, 2, 4])).sum(1).astype(np.uint8)).cuda()
    grid, mp, L = _abi.Grid(*n, *l), _abi.MatProp(E, nu, 0.0, 0.0, 1.0), _abi.lib()
    assert L.vfgpu_set_u_split(ctx.h, 7) != 0  # not a mode
    xd = torch.from_numpy(x).cuda()
    for v in (blob, rng.uniform(0, 1, o.N), np.ones(o.N), blob):
        ctx.set_field("V", v)
        ctx.set_u_split("off")
        y1, y1_32 = ctx.u_apply(xd, vg.FP64).cpu().numpy(), ctx.u_apply(x, vg.MIXED)
        ctx.set_u_split("on")
        y = ctx.u_apply(xd, vg.FP64).cpu().numpy()
        assert np.array_equal(y, y1)
        assert np.array_equal(ctx.u_apply(x, vg.MIXED), y1_32)
        assert np.array_equal(ctx.u_apply(x, vg.FP64), y)
        vd, yna = torch.from_numpy(v).cuda(), torch.full_like(xd, float("nan"))
        torch.cuda.synchronize()
        rc = L.vfgpu_u_apply_noalloc(C.byref(grid), C.byref(mp), eta, vd.data_ptr(), bits.data_ptr(),
                                     xd.data_ptr(), yna.data_ptr(), None)
        assert rc == 0, L.vfgpu_last_error().decode()
        torch.cuda.synchronize()
        assert np.array_equal(yna.cpu().numpy(), y)
        yref = o.u_apply(v, x, mask)
        assert np.abs(y - yref).max() <= 1e-12 * np.abs(yref).max()
        y32 = ctx.u_apply(x, vg.MIXED)
        assert np.linalg.norm(y32 - yref) <= 2e-6 * np.linalg.norm(yref)
    ctx.close()


@pytest.mark.parametrize("n,l", [((1025, 513, 3), (4.0, 2.0, 2.0 / 256)),   # cubic cells
                                 ((1025, 1041, 3), (4.0, 3.0, 0.05))])
def test_unit_lists_column_limit(cuda, oracle_mod, n, l):
    """The one-block list builder takes up to 2048 tile columns per plan.  At 1025 x 513 x 3
    the FP64 plan (32 x 8 element tiles) has exactly 2048 columns and the FP32 one (32 x 16)
    1024: both split.  At 1025 x 1041 x 3 both are past the limit (4160 / 2080 columns) and
    keep one wave although the split is asked for.  Either way: the bits of one wave (FP64
    and FP32) and of the fixed-scratch apply, and the oracle's values (FP64 1e-12, FP32
    2e-6), on a field with intact, constant-damage and random regions."""
    import ctypes as C

    import vpfhf_b200 as vg
    from vpfhf_b200 import _abi
    torch = cuda
    E, nu, eta = 1e10, 0.25, 1e-8
    o = oracle_mod.Oracle(n, l, E=E, nu=nu, eta=eta)
    ctx = vg.VFContext(n, l, dict(E=E, nu=nu), eta=eta)
    ctx.set_bc(vg.rollers())
    mask, _ = o.bc(oracle_mod.rollers_face())
    rng = np.random.default_rng(11)
    v = np.ones(o.N)
    vv = v.reshape(n[2], n[1], n[0])
    y0, y1 = n[1] // 5, n[1] // 3
    vv[:, y0:y1, 300:520] = rng.uniform(0, 1, (n[2], y1 - y0, 220))
    vv[1:, -n[1] // 4:, :40] = 0.3
    ctx.set_field("V", v)
    x = rng.standard_normal(3 * o.N) * 1e-3
    xd = torch.from_numpy(x).cuda()
    ctx.set_u_split("off")
    y_one, y_one32 = ctx.u_apply(xd, vg.FP64).cpu().numpy(), ctx.u_apply(x, vg.MIXED)
    ctx.set_u_split("on")
    y = ctx.u_apply(xd, vg.FP64).cpu().numpy()
    assert np.array_equal(y, y_one)
    y32 = ctx.u_apply(x, vg.MIXED)
    assert np.array_equal(y32, y_one32)
    bits = torch.from_numpy((mask.reshape(o.N, 3) * np.array([1, 2, 4])).sum(1).astype(np.uint8)).cuda()
    vd, yna = torch.from_numpy(v).cuda(), torch.full_like(xd, float("nan"))
    L = _abi.lib()
    torch.cuda.synchronize()
    rc = L.vfgpu_u_apply_noalloc(C.byref(_abi.Grid(*n, *l)), C.byref(_abi.MatProp(E, nu, 0.0, 0.0, 1.0)), eta,
                                 vd.data_ptr(), bits.data_ptr(), xd.data_ptr(), yna.data_ptr(), None)
    assert rc == 0, L.vfgpu_last_error().decode()
    torch.cuda.synchronize()
    assert np.array_equal(yna.cpu().numpy(), y)
    yref = o.u_apply(v, x, mask)
    assert np.abs(y - yref).max() <= 1e-12 * np.abs(yref).max()
    assert np.linalg.norm(y32 - yref) <= 2e-6 * np.linalg.norm(yref)
    ctx.close()


def test_u_operator_properties_161(cuda, oracle_mod):
    """161^3 (16.7M U dofs: past the oracle's sizes) with a penny crack, a constant block
    and a random block of v, the applies split by phase field (AUTO at this size):
    on vectors that vanish on the Dirichlet dofs the operator is symmetric (1e-12) and
    positive, it is linear (1e-13), one wave gives the same bits, and FP32 stays within
    2e-6 of FP64 normwise."""
    import vpfhf_b200 as vg
    torch = cuda
    n, l = (161, 161, 161), (4.0, 4.0, 4.0)
    o = oracle_mod.Oracle(n, l, epsilon=2 * 4.0 / 160)
    mask, _ = o.bc(oracle_mod.rollers_face())
    free = mask == 0
    v = o.penny_v((2.0, 2.0, 2.0), 0.8)
    vv = v.reshape(n[2], n[1], n[0])
    rng = np.random.default_rng(12)
    vv[:20, :20, :20] = 0.4
    vv[-12:, -12:, -12:] = rng.uniform(0, 1, (12, 12, 12))
    ctx = vg.VFContext(n, l, dict(E=1e10, nu=0.25), eta=1e-8)
    ctx.set_bc(vg.rollers())
    ctx.set_field("V", vv.reshape(-1).copy())
    x, y = (rng.standard_normal(3 * o.N) * free for _ in range(2))
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    ax = ctx.u_apply(xd, vg.FP64)
    ay = ctx.u_apply(yd, vg.FP64)
    axy = ctx.u_apply(2.0 * xd - 3.0 * yd, vg.FP64)
    xay, yax = float(torch.dot(xd, ay)), float(torch.dot(yd, ax))
    assert abs(xay - yax) <= 1e-12 * max(abs(xay), abs(yax))
    assert float(torch.dot(xd, ax)) > 0 and float(torch.dot(yd, ay)) > 0
    lin = axy - (2.0 * ax - 3.0 * ay)
    assert float(lin.norm()) <= 1e-13 * float(axy.norm())
    ctx.set_u_split("off")
    assert torch.equal(ctx.u_apply(xd, vg.FP64), ax)
    ctx.set_u_split("auto")
    a32 = ctx.u_apply(xd, vg.MIXED)
    assert float((a32 - ax).norm()) <= 2e-6 * float(ax.norm())
    ctx.close()


def test_layered_material_split(cuda, oracle_mod):
    """Three material layers across z (per-element-layer Lame coefficients in the device
    parameter block) with a mostly intact phase field: the applies split by phase field
    and in one wave give the same bits, FP64 at 1e-12 and FP32 at 2e-6 against the
    oracle."""
    import vpfhf_b200 as vg
    n, l = (45, 37, 33), (2.0, 1.6, 1.4)
    E, nu = [1e10, 3e10, 0.6e10], [0.25, 0.3, 0.2]
    layer = np.array([0] * 10 + [1] * 12 + [2] * 10, np.int32)  # nz - 1 element layers
    o = oracle_mod.Oracle(n, l, E=E, nu=nu, eta=1e-8, layer=layer)
    mask, _ = o.bc(oracle_mod.rollers_face())
    rng = np.random.default_rng(14)
    v = np.ones(o.N)
    vv = v.reshape(n[2], n[1], n[0])
    vv[12:20, 5:20, 3:30] = rng.uniform(0, 1, vv[12:20, 5:20, 3:30].shape)
    vv[25:, :, :] = 0.5
    ctx = vg.VFContext(n, l, [dict(E=e, nu=p) for e, p in zip(E, nu)], eta=1e-8, layer=layer)
    ctx.set_bc(vg.rollers())
    ctx.set_field("V", v)
    x = rng.standard_normal(3 * o.N) * 1e-3
    xd = cuda.from_numpy(x).cuda()
    yref = o.u_apply(v, x, mask)
    ys = {}
    for split in ("off", "on"):
        ctx.set_u_split(split)
        ys[split] = (ctx.u_apply(xd, vg.FP64).cpu().numpy(), ctx.u_apply(x, vg.MIXED))
    assert np.array_equal(ys["on"][0], ys["off"][0]) and np.array_equal(ys["on"][1], ys["off"][1])
    assert np.abs(ys["on"][0] - yref).max() <= 1e-12 * np.abs(yref).max()
    assert np.linalg.norm(ys["on"][1] - yref) <= 2e-6 * np.linalg.norm(yref)
    ctx.close()
