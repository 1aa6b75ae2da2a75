"""GPU: StepU with the geometric multigrid preconditioner (solve option pc="mg").

The multigrid PCG has no counterpart in the reference (whose snesU runs KSPCG with
Jacobi, VFCommon.c:1044-1047); it stops at the same Jacobi-preconditioned residual,
so its Newton solutions match the oracle's StepU and the Jacobi solve on the GPU,
with far fewer Krylov iterations."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _penny_ctx(n, L=4.0, cellE=None):
    import vpfhf_b200 as vg
    shape = (n, n, n) if np.isscalar(n) else tuple(n)
    h = max(L / (m - 1) for m in shape)
    ctx = vg.VFContext(shape, (L, L, L), dict(E=1e10, nu=0.25, Gc=100.0), epsilon=2 * h,
                       eta=1e-8, atnum=1, pressurize=True)
    ctx.set_bc(vg.rollers())
    ctx.set_field("pressure", np.full(ctx.N, 1e6))
    if cellE is not None:
        ctx.set_cell_modulus(cellE)
    ctx.init_cracks([dict(center=(L / 2, L / 2, L / 2), r=0.2 * L, theta=30.0, phi=20.0,
                          thickness=2 * h)])
    ctx.time_step_prepare()
    return ctx


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mg_matches_oracle_step_u(cuda, oracle_mod, precision):
    """17^3 penny (levels 17, 9, 5), V-cycle in FP64 or FP32: U and energies against the
    oracle's Jacobi StepU."""
    import vpfhf_b200 as vg
    n, L = 17, 4.0
    h = L / (n - 1)
    kw = dict(E=1e10, nu=0.25, Gc=100.0, epsilon=2 * h, eta=1e-8, atnum=1)
    o = oracle_mod.Oracle((n, n, n), (L, L, L), pressurize=True, **kw)
    v = o.penny_v((2.0, 2.0, 2.0), 0.8)
    p = np.full(o.N, 1e6)
    mask, val = o.bc(oracle_mod.rollers_face())
    u = np.zeros(3 * o.N)
    assert o.step_u(u, v, p=p, mask=mask, value=val).reason > 0
    ctx = vg.VFContext((n, n, n), (L, L, L), dict(E=kw["E"], nu=kw["nu"], Gc=kw["Gc"]),
                       epsilon=kw["epsilon"], eta=kw["eta"], atnum=1, pressurize=True)
    ctx.set_bc(vg.rollers())
    ctx.set_field("V", v)
    ctx.set_field("VIrrev", v)
    ctx.set_field("pressure", p)
    rc, st = ctx.step_u(dict(pc="mg", precision=precision))
    assert rc == 0 and st["reason"] > 0, st
    ug = ctx.get_field("U")
    assert np.linalg.norm(ug - u) <= 1e-6 * np.linalg.norm(u)
    el, _, pw = ctx.u_energy()
    el_o, pw_o = o.u_energy(u, v, p=p)
    assert el == pytest.approx(el_o, rel=1e-7) and pw == pytest.approx(pw_o, rel=1e-7)
    ctx.close()


@pytest.mark.parametrize("hetero,precision,split", [(False, "fp64", "auto"), (True, "fp64", "auto"),
                                                   (True, "mixed", "auto"), (True, "fp64", "on"),
                                                   (True, "mixed", "on")])
def test_mg_matches_jacobi_65(cuda, hetero, precision, split):
    """65^3 inclined penny, uniform or log-normal per-cell modulus: the multigrid (FP64 or
    FP32 V-cycle) and the FP64 Jacobi StepU reach the same U, the multigrid in a tenth of
    the Krylov iterations; with the U applies in one wave (auto at this size) and split
    by phase field (on: the Jacobi CG's fused p.w, the V-cycle's fine level and the
    multigrid's outer FP64 applies on the two waves)."""
    n = 65
    cellE = None
    if hetero:
        rng = np.random.default_rng(5)
        cellE = (1e10 * np.exp(0.5 * rng.standard_normal((n - 1) ** 3))).astype(np.float32)
    res = {}
    for pc in ("jacobi", "mg"):
        ctx = _penny_ctx(n, cellE=cellE)
        ctx.set_u_split(split)
        rc, st = ctx.step_u(dict(pc=pc, precision=precision if pc == "mg" else "fp64"))
        assert rc == 0 and st["reason"] > 0, (pc, st)
        res[pc] = (ctx.get_field("U"), st, ctx.u_energy())
        ctx.close()
    uj, sj, ej = res["jacobi"]
    um, sm, em = res["mg"]
    assert np.linalg.norm(um - uj) <= 1e-6 * np.linalg.norm(uj)
    assert em[0] == pytest.approx(ej[0], rel=1e-8) and em[2] == pytest.approx(ej[2], rel=1e-8)
    assert sm["ksp_its"] * 10 <= sj["ksp_its"], (sm, sj)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mg_nocompression_newton(cuda, oracle_mod, precision):
    """The squeezed NOCOMPRESSION crack (13^3: levels 13, 7): the multigrid preconditions
    the re-formed Jacobian of every Newton step and lands on the oracle's solution."""
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
    assert o.step_u(uo, v, mask=mask, value=val).reason > 0
    bc = [vg.BCSpec(X0=vg.BC_ZERO, X1=vg.BC_ZERO), vg.BCSpec(Y0=vg.BC_ZERO, Y1=vg.BC_ZERO),
          vg.BCSpec(Z0=vg.BC_ZERO, Z1=(vg.BC_FIXED, -0.01))]
    ctx.set_bc(bc)
    ctx.set_field("BCU", bcu)
    ctx.time_step_prepare()
    rc, s = ctx.step_u(dict(pc="mg", precision=precision))
    assert rc == 0 and s["reason"] > 0 and s["newton_its"] >= 2, s
    ug = ctx.get_field("U")
    assert np.linalg.norm(ug - uo) <= 1e-6 * np.linalg.norm(uo)
    ctx.close()


@pytest.mark.parametrize("shape,cells", [((48, 48, 48), False), ((40, 33, 12), True)])
def test_mg_any_grid(cuda, shape, cells):
    """Odd cell counts and unequal axes: 48^3 nodes (levels 48, 25, 13, 7: non-nested
    transfers on every level) and 40 x 33 x 12 nodes with a per-cell modulus (levels
    (40,33,12), (21,17,7), (11,9,7), (6,5,7): anisotropic coarse cells, an axis that stops
    coarsening).  The FP32 V-cycle multigrid reaches the FP64 Jacobi solution in a fifth
    of the Krylov iterations."""
    cellE = None
    if cells:
        rng = np.random.default_rng(11)
        nc = int(np.prod([m - 1 for m in shape]))
        cellE = (1e10 * np.exp(0.5 * rng.standard_normal(nc))).astype(np.float32)
    res = {}
    for pc in ("jacobi", "mg"):
        ctx = _penny_ctx(shape, cellE=cellE)
        rc, st = ctx.step_u(dict(pc=pc, precision="mixed" if pc == "mg" else "fp64"))
        assert rc == 0 and st["reason"] > 0, (pc, st)
        res[pc] = (ctx.get_field("U"), st, ctx.u_energy())
        ctx.close()
    uj, sj, ej = res["jacobi"]
    um, sm, em = res["mg"]
    assert np.linalg.norm(um - uj) <= 1e-6 * np.linalg.norm(uj)
    assert em[0] == pytest.approx(ej[0], rel=1e-8) and em[2] == pytest.approx(ej[2], rel=1e-8)
    assert sm["ksp_its"] * 5 <= sj["ksp_its"], (sm, sj)


def test_mg_rejected_cases(cuda):
    """A grid with fewer than 9 nodes along every axis (no coarse grid) is refused with
    VFGPU_ERR_INVALID in both precisions; the context stays usable for a Jacobi solve."""
    import vpfhf_b200 as vg
    ctx = _penny_ctx(8)
    with pytest.raises(vg.VFGPUError) as ei:
        ctx.step_u(dict(pc="mg"))
    assert ei.value.code == -1 and "multigrid" in str(ei.value)
    with pytest.raises(vg.VFGPUError) as ei:
        ctx.step_u(dict(pc="mg", precision="mixed"))
    assert ei.value.code == -1
    rc, st = ctx.step_u()
    assert rc == 0 and st["reason"] > 0, st
    ctx.close()


def test_mg_precision_switch_and_am_loop(cuda):
    """One context alternating FP64 and FP32 V-cycles (the hierarchy is rebuilt on each
    switch) through AM steps: each result is bit-identical to a fresh context's."""
    n = 33

    def run(ctx, precisions):
        out = []
        for prec in precisions:
            rc, err, su, sv = ctx.am_step(dict(pc="mg", precision=prec))
            assert rc == 0, (su, sv)
            out.append((ctx.get_field("U"), ctx.get_field("V")))
        return out

    a = _penny_ctx(n)
    got = run(a, ["fp64", "mixed", "fp64"])
    a.close()
    for k, prec in enumerate(["fp64", "mixed", "fp64"]):
        b = _penny_ctx(n)
        ref = run(b, ["fp64", "mixed", "fp64"][:k + 1])[-1]
        b.close()
        assert np.array_equal(got[k][0], ref[0]) and np.array_equal(got[k][1], ref[1]), prec


@pytest.mark.parametrize("n,resolved", [(33, "jacobi"), (65, "mg")])
def test_auto_preconditioner_resolves_by_grid(cuda, n, resolved):
    """pc="auto" is the Jacobi solve below 65 nodes per axis and the multigrid one from
    65 on: the same bits as the solve it resolves to."""
    out = {}
    for pc in ("auto", resolved):
        ctx = _penny_ctx(n)
        rc, st = ctx.step_u(dict(pc=pc, precision="mixed"))
        assert rc == 0 and st["reason"] > 0, st
        out[pc] = (ctx.get_field("U"), st["ksp_its"])
        ctx.close()
    assert np.array_equal(out["auto"][0], out[resolved][0])
    assert out["auto"][1] == out[resolved][1]
