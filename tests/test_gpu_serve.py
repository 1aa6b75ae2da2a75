"""GPU: device crack initialisers against the oracle, and the serving loop -- results
against a direct solve and the oracle, and the same bits alone and in a mix."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PENNIES = [dict(center=(2.0, 2.0, 2.0), r=0.8, theta=0.0, phi=0.0, thickness=0.0),
           dict(center=(1.3, 2.6, 1.9), r=0.55, theta=35.0, phi=62.0, thickness=0.05),
           dict(center=(2.7, 1.2, 2.4), r=0.0, theta=0.0, phi=0.0, thickness=0.0)]
RECTS = [dict(corners=(1.0, 1.0, 2.5, 3.0, 1.2, 2.5, 1.1, 3.0, 2.7), thickness=0.1),
         dict(corners=(0.5, 2.0, 0.5, 0.5, 3.5, 0.5, 0.5, 2.0, 3.5), thickness=0.0)]


def _rows(pennies, rects):
    pr = [list(p["center"]) + [p["r"], p["theta"], p["phi"], p["thickness"]] for p in pennies]
    rr = [list(r["corners"]) + [r["thickness"]] for r in rects]
    return pr, rr


@pytest.mark.parametrize("atnum", [1, 2])
@pytest.mark.parametrize("with_rects", [False, True])
def test_device_cracks_match_oracle(cuda, oracle_mod, atnum, with_rects):
    import vpfhf_b200 as vg
    n, L, eps = (33, 29, 25), (4.0, 4.0, 4.0), 0.25
    rects = RECTS if with_rects else []
    o = oracle_mod.Oracle(n, L, E=1e10, nu=0.25, Gc=100.0, epsilon=eps, eta=1e-8, atnum=atnum)
    pr, rr = _rows(PENNIES, rects)
    ref = o.cracks_v(pennies=pr, rects=rr)
    ctx = vg.VFContext(n, L, dict(E=1e10, nu=0.25, Gc=100.0), epsilon=eps, eta=1e-8, atnum=atnum)
    ctx.init_cracks(PENNIES, rects)
    v, vi = ctx.get_field("V"), ctx.get_field("VIrrev")
    assert np.array_equal(v, vi)
    # penny AT1 is plain arithmetic (bit for bit up to libm's pow(x, 2)); the AT2
    # exponential and the rectangle's acos / sin differ from the host libm by ulps
    tol = 1e-15 if (atnum == 1 and not with_rects) else 1e-12
    assert np.abs(v - ref).max() <= tol
    assert (v == 0).sum() == (ref == 0).sum()
    # no cracks: V = VIrrev = 1; more than one batch of cracks (> 16)
    ctx.init_cracks()
    assert np.array_equal(ctx.get_field("V"), np.ones(ctx.N))
    many = [dict(center=(0.2 + 0.2 * k, 2.0, 2.0), r=0.3, theta=10.0 * k, phi=45.0, thickness=0.0)
            for k in range(19)]
    ctx.init_cracks(many)
    pr, _ = _rows(many, [])
    assert np.abs(ctx.get_field("V") - o.cracks_v(pennies=pr)).max() <= 1e-12
    ctx.close()


def _oracle_am(oracle_mod, p, its):
    """The oracle's AM loop for a pressurised-crack problem on rollers: AT1 bounds
    [0, VIrrev]; AT2 bounds [0, 1] with the nodes whose VIrrev <= irrevtol pinned."""
    o = oracle_mod.Oracle(p.n, p.l, E=p.E, nu=p.nu, Gc=p.Gc, epsilon=p.eps, eta=p.eta,
                          atnum=p.atnum, pressurize=True)
    pr, rr = _rows(p.pennies, p.rects)
    V = o.cracks_v(pennies=pr, rects=rr)
    U = np.zeros(3 * o.N)
    pres = np.full(o.N, p.pressure)
    umask, uval = o.bc(oracle_mod.rollers_face())
    virrev = V.copy()
    lb, ub = np.zeros(o.N), (virrev.copy() if p.atnum == 1 else np.ones(o.N))
    for _ in range(its):
        o.step_u(U, V, p=pres, mask=umask, value=uval)
        o.step_v(V, U, lb, ub, p=pres, virrev=virrev if p.atnum == 2 else None)
    el, pw = o.u_energy(U, V, p=pres)
    return dict(elastic=el, pressure_work=pw, surface=o.v_energy(V), cov=o.cov(U, V)), V


@pytest.mark.parametrize("atnum", [1, 2])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_server_matches_direct_and_oracle(cuda, oracle_mod, precision, atnum):
    import vpfhf_b200 as vg
    from vpfhf_b200.serve import Problem, Server
    p = Problem(n=(17, 17, 17), E=1.2e10, nu=0.22, atnum=atnum, pennies=PENNIES[:2], am_its=3,
                precision=precision)
    vs = np.empty(p.nodes)
    with Server(workers=2) as srv:
        srv.submit(p, out_v=vs)
        r = srv.next(120.0)
    assert r is not None and r["status"] >= 0, r
    assert r["am_its"] == 3
    # the same problem through a VFContext: the same kernels, so the same bits
    ctx = vg.VFContext(p.n, p.l, dict(E=p.E, nu=p.nu, Gc=p.Gc), epsilon=p.eps, eta=p.eta,
                       atnum=p.atnum, pressurize=True)
    ctx.set_bc(vg.rollers())
    ctx.set_field("pressure", np.full(ctx.N, p.pressure))
    ctx.init_cracks(p.pennies)
    ctx.time_step_prepare()
    for _ in range(3):
        ctx.am_step(dict(precision=precision))
    el, _, pw = ctx.u_energy()
    assert (r["elastic"], r["pressure_work"], r["surface"], r["cov"]) == \
        (el, pw, ctx.v_energy(), ctx.crack_opening())
    assert np.array_equal(vs, ctx.get_field("V"))
    ctx.close()
    # and the oracle, at the parity bar (relative energy 1e-6, V L-inf 1e-4)
    ref, vref = _oracle_am(oracle_mod, p, 3)
    for k in ("elastic", "pressure_work", "surface", "cov"):
        assert r[k] == pytest.approx(ref[k], rel=1e-6), k
    assert np.abs(vs - vref).max() <= 1e-4


def _mix(n_extra=12, seed=7):
    from vpfhf_b200.serve import serving_stream
    probes = serving_stream(count=4, seed=11, edges=(17, 33), am_its=2)
    for k, p in enumerate(probes):
        p.tag = 1000 + k
        p.precision = "mixed" if k % 2 else "fp64"
    extra = serving_stream(count=n_extra, seed=seed, edges=(17, 33), am_its=2)
    return probes, extra


def test_results_same_alone_and_in_the_mix(cuda):
    """Each probe problem alone on an idle server, then inside a stream of other problems
    on 4 workers (pooled contexts reused across problems, graphs kept), then on a memory
    budget so tight that problems wait for memory and contexts are evicted: identical bits
    every time."""
    from vpfhf_b200.serve import Server
    probes, extra = _mix()
    alone = {}
    for p in probes:
        v = np.empty(p.nodes)
        with Server(workers=1) as srv:
            srv.submit(p, out_v=v)
            r = srv.next(300.0)
        assert r["status"] >= 0, r
        assert r["reused_ctx"] == 0
        alone[p.tag] = (r, v)

    def run_mix(budget):
        order = extra[:6] + probes[:2] + extra[6:] + probes[2:]
        vs = {p.tag: np.empty(p.nodes) for p in probes}
        got = {}
        with Server(workers=4, budget_bytes=budget) as srv:
            for p in order:
                srv.submit(p, out_v=vs.get(p.tag))
            for _ in order:
                r = srv.next(600.0)
                assert r is not None and r["status"] >= 0, r
                got[r["tag"]] = r
            info = srv.info()
        return got, vs, info

    from vpfhf_b200 import _abi
    import ctypes
    b = ctypes.c_longlong()
    _abi.lib().vfgpu_memory_estimate(ctypes.byref(_abi.Grid(33, 33, 33, 4., 4., 4.)), ctypes.byref(b))
    # 1.05x one 33^3 ctx: a 33^3 and a 17^3 ctx never fit together, so every switch of
    # grid size with the other ctx idle evicts it
    for budget, check_pool in ((0, "reuse"), (int(1.05 * b.value), "evict")):
        got, vs, info = run_mix(budget)
        if check_pool == "reuse":
            assert sum(r["reused_ctx"] for r in got.values()) > 0
        else:
            assert info["evictions"] > 0 and info["peak_reserved_bytes"] <= budget
        for p in probes:
            ra, va = alone[p.tag]
            rm = got[p.tag]
            for k in ("elastic", "pressure_work", "surface", "cov", "am_err", "ksp_its_u",
                      "ksp_its_v"):
                assert rm[k] == ra[k], (p.tag, k, budget)
            assert np.array_equal(vs[p.tag], va), (p.tag, budget)


def test_multigrid_problems_in_the_mix(cuda):
    """Multigrid-preconditioned problems (FP64 and FP32 V-cycles) served among Jacobi ones
    on 3 workers: each result has the bits it has alone, and matches the Jacobi solve of
    the same problem to the solver tolerance."""
    import dataclasses
    from vpfhf_b200.serve import Server, serving_stream
    base = serving_stream(count=9, seed=77, edges=(17, 33, 65), am_its=3)
    probs = []
    for i, p in enumerate(base):
        pc, prec = (("mg", "fp64"), ("mg", "mixed"), ("jacobi", "fp64"))[i % 3]
        probs.append(dataclasses.replace(p, pc=pc, precision=prec, tag=i))
    alone = {}
    for p in probs[:6]:
        with Server(workers=1) as srv:
            srv.submit(p)
            r = srv.next(300.0)
        assert r["status"] >= 0, r
        alone[p.tag] = r
    with Server(workers=3) as srv:
        for p in probs:
            srv.submit(p)
        got = {}
        for _ in probs:
            r = srv.next(600.0)
            assert r is not None and r["status"] >= 0, r
            got[r["tag"]] = r
    for tag, ra in alone.items():
        for k in ("elastic", "pressure_work", "surface", "cov", "am_err", "ksp_its_u"):
            assert got[tag][k] == ra[k], (tag, k)
    # against the Jacobi solve of the same problems
    with Server(workers=2) as srv:
        for p in probs[:6]:
            srv.submit(dataclasses.replace(p, pc="jacobi", precision="fp64"))
        jac = {}
        for _ in range(6):
            r = srv.next(600.0)
            jac[r["tag"]] = r
    for tag, ra in alone.items():
        if probs[tag].pc != "mg":
            continue
        for k in ("elastic", "pressure_work", "surface", "cov"):
            assert ra[k] == pytest.approx(jac[tag][k], rel=1e-6), (tag, k)
        assert ra["ksp_its_u"] * 5 < jac[tag]["ksp_its_u"], tag


def test_server_errors(cuda):
    from vpfhf_b200 import VFGPUError
    from vpfhf_b200.serve import Problem, Server
    with Server(workers=2, budget_bytes=1 << 20) as srv:
        # too large for the budget: the result carries VFGPU_ERR_OOM, the server goes on
        srv.submit(Problem(n=(33, 33, 33), pennies=PENNIES[:1], am_its=1, tag=1))
        r = srv.next(60.0)
        assert r["status"] == -3 and "budget" in r["error"]
        with pytest.raises(VFGPUError):
            srv.submit(Problem(n=(1, 17, 17), epsilon=0.5, am_its=1))
        with pytest.raises(VFGPUError):
            srv.submit(Problem(n=(17, 17, 17), am_its=0, max_am_its=0))
        assert srv.next(0.01) is None
