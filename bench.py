"""Benchmark of the U operator (matvec GDOF/s) and the AM step on the 129^3
pressurized penny crack (the FP64-vs-mixed configuration), one JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A "step" is one application of the degraded elasticity operator K(v) to a
3N-vector (3 x 129^3 = 6,440,067 dofs) with the inputs resident in HBM; the L2
is flushed between timed steps.  `e2e` times the same step through the C ABI
(vfgpu_u_apply) from pinned host memory, copies included (the entry point overlaps the
copies in both directions with the apply, slab by slab).  The AM-step rate
(StepU + StepV to tolerance, FP64 and mixed, 10 iterations from the penny-crack
start; U solve with the reference's Jacobi PCG and with the multigrid PCG) is
reported beside it with the mixed-vs-FP64 differences of the energies,
the crack opening and V, and so is the serving stream (p50 / p99 latency and
throughput of independent problems through the library's request loop).

Multi-GPU: the operator does not shard in this build ("replicas only"): every
rank runs its own copy of the workload and `value` is the total over ranks.

--impl reference times the reference's CPU algorithm for the same metric: the
assembled AIJ (CSR, 81 nnz/row) sparse matrix-vector product that KSPCG runs
(restated in the oracle, oracle/vf_oracle.c) on all host cores, on the same 129^3
workload, and beside it the AM step by the reference's method (assembled Jacobians,
CG on the assembled matrix) on the 41^3 penny crack.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_EDGE, L_BOX = 129, 4.0
# AM-step variants: (key, precision, U preconditioner)
AM_VARIANTS = (("fp64", "fp64", "jacobi"), ("mixed", "mixed", "jacobi"),
               ("mg_fp64", "fp64", "mg"), ("mg_mixed", "mixed", "mg"))
WORKLOAD = "penny crack 129^3 (6.44M U dofs), E=1e10 nu=0.25 Gc=100 AT1 eps=2h eta=1e-8 p=1e6"


def _rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(vals, dist=None, device="cpu"):
    """Element-wise maximum of a list of times over the ranks (the slowest rank sets
    every timed number); identity without a process group."""
    if dist is None:
        return [float(v) for v in vals]
    import torch
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while active."""

    def __init__(self, gpu):
        self.gpu, self.proc, self.path = gpu, None, None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except Exception:
            pass
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def setup_problem(vg, n):
    """The 129^3 penny crack at its first AM iterate (v from VFPennyCrackBuildVAT1)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    h = L_BOX / (n - 1)
    ctx = vg.VFContext((n, n, n), (L_BOX,) * 3, dict(E=1e10, nu=0.25, Gc=100.0), epsilon=2 * h,
                       eta=1e-8, atnum=1, pressurize=True)
    ctx.set_bc(vg.rollers())
    v0 = vg.penny_crack_v((n, n, n), (L_BOX,) * 3, (L_BOX / 2,) * 3, 0.4, epsilon=2 * h)
    ctx.set_field("V", v0)
    ctx.set_field("pressure", np.full(ctx.N, 1e6))
    ctx.time_step_prepare()
    return ctx, v0


def fp_peak_tflops(torch, dtype):
    """Measured FMA throughput of the CUDA cores (a dependent-chain-free FMA kernel)."""
    from vpfhf_b200 import _abi
    import ctypes as C
    L = _abi.lib()
    if not hasattr(L, "vfgpu_fma_peak"):
        return None
    L.vfgpu_fma_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    L.vfgpu_fma_peak.restype = C.c_int
    out = C.c_double()
    if L.vfgpu_fma_peak(8 if dtype == "f64" else 4, C.byref(out)) != 0:
        return None
    return out.value


def run_gpu(args):
    import torch
    import vpfhf_b200 as vg

    rank, world, local = _rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    n = args.grid
    ctx, v0 = setup_problem(vg, n)
    N3 = 3 * ctx.N
    s = ctx.torch_stream()
    rng = np.random.default_rng(1000 + rank)
    x_host = rng.standard_normal(N3) * 1e-4
    x = torch.from_numpy(x_host).cuda()
    y = torch.empty_like(x)
    x32, y32 = x.float(), torch.empty(N3, dtype=torch.float32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    torch.cuda.synchronize()

    def timed_applies(prec, xi, yi, K, W):
        for _ in range(W):
            ctx.u_apply_dev(xi, yi, prec)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(K)]
        barrier()
        for a, b in ev:
            with torch.cuda.stream(s):
                flush.zero_()
            a.record(s)
            ctx.u_apply_dev(xi, yi, prec)
            b.record(s)
        torch.cuda.synchronize()
        barrier()
        return [a.elapsed_time(b) for a, b in ev]

    with ClockSampler(local) as clk:
        t64 = timed_applies(vg.FP64, x, y, args.steps, args.warmup)
    clocks = clk.summary()
    t32 = timed_applies(vg.MIXED, x32, y32, args.steps, args.warmup)
    ms64 = float(np.mean(t64))
    ms32 = float(np.mean(t32))
    # the tensor-core element contraction (vfgpu_u_apply_tc), same FP32 inputs
    mstc, tc_ok = float("nan"), False
    for _ in range(args.warmup if args.tc else 0):
        ctx.u_apply_tc(x32, y32)
    if args.tc:
        evt = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        barrier()
        for a, b in evt:
            with torch.cuda.stream(s):
                flush.zero_()
            a.record(s)
            ctx.u_apply_tc(x32, y32)
            b.record(s)
        torch.cuda.synchronize()
        mstc = float(np.mean([a.elapsed_time(b) for a, b in evt]))
        tc_ok = not ctx.tc_error()
    ms64, ms32, mstc = max_over_ranks([ms64, ms32, mstc], dist, "cuda")

    if args.only_am:
        out = {}
        for prec in ("fp64", "mixed"):
            ctx.set_field("U", np.zeros(N3))
            ctx.set_field("V", v0)
            ctx.time_step_prepare()
            steps = []
            for it in range(args.am_steps):
                last = it == args.am_steps - 1
                barrier()
                if last and prec == args.profile_precision:
                    torch.cuda.profiler.start()
                t0 = time.perf_counter()
                rc, err, su, sv = ctx.am_step(dict(precision=prec, pc=args.am_pc))
                barrier()
                dt = time.perf_counter() - t0
                if last and prec == args.profile_precision:
                    torch.cuda.profiler.stop()
                steps.append(dict(s=dt, u_s=su["seconds"], v_s=sv["seconds"],
                                  u_newton=su["newton_its"], u_ksp=su["ksp_its"],
                                  u_refine=su["refine_its"], v_newton=sv["newton_its"],
                                  v_ksp=sv["ksp_its"], v_refine=sv["refine_its"], err=err))
            out[prec] = steps
        if rank == 0:
            print(json.dumps({"grid": n, "pc": args.am_pc, "am": out}))
        ctx.close()
        if dist:
            dist.destroy_process_group()
        return

    if args.only_apply:
        if rank == 0:
            print(json.dumps({"grid": n, "ms_fp64": ms64, "ms_fp32": ms32, "ms_tc": mstc,
                              "tc_ok": tc_ok, "clocks": clocks}))
        ctx.close()
        if dist:
            dist.destroy_process_group()
        return

    # e2e through the C ABI from pinned host memory (H2D of x, D2H of y every step)
    xp = torch.empty(N3, dtype=torch.float64, pin_memory=True)
    xp.numpy()[:] = x_host
    yp = torch.empty(N3, dtype=torch.float64, pin_memory=True)
    xpn, ypn = xp.numpy(), yp.numpy()
    for _ in range(args.warmup):
        ctx.u_apply(xpn, vg.FP64, out=ypn)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.u_apply(xpn, vg.FP64, out=ypn)
    barrier()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    (e2e_ms,) = max_over_ranks([e2e_ms], dist, "cuda")

    # AM steps (StepU + StepV to tolerance) from the penny-crack start: FP64 and mixed,
    # with the reference's Jacobi-preconditioned U solve and with the multigrid one
    am, vfin = {}, {}
    for key, prec, pc in AM_VARIANTS:
        ctx.set_field("U", np.zeros(N3))
        ctx.set_field("V", v0)
        ctx.time_step_prepare()
        times, energies = [], []
        for it in range(args.am_steps):
            barrier()
            t0 = time.perf_counter()
            rc, err, su, sv = ctx.am_step(dict(precision=prec, pc=pc))
            barrier()
            times.append(time.perf_counter() - t0)
            el, _, pw = ctx.u_energy()
            energies.append((el, pw, ctx.v_energy(), ctx.crack_opening()))
        am[key] = dict(s_per_step=float(np.mean(times[1:] if len(times) > 1 else times)),
                       energies=energies, last_kspU=su["ksp_its"], last_kspV=sv["ksp_its"])
        vfin[key] = ctx.get_field("V")
    names = ("elastic", "pressure_work", "surface", "cov")

    def versus_fp64(key):  # against the FP64 Jacobi run (the reference's solve)
        rel = max(abs(a - b) / abs(b) for ea, eb in zip(am[key]["energies"], am["fp64"]["energies"])
                  for a, b in zip(ea, eb))
        rel_last = {k: abs(a - b) / abs(b) for k, a, b in
                    zip(names, am[key]["energies"][-1], am["fp64"]["energies"][-1])}
        return rel, rel_last, float(np.abs(vfin[key] - vfin["fp64"]).max())
    rel, rel_last, v_linf = versus_fp64("mixed")
    vs_oracle = versus_oracle(am, vfin, n, args.am_steps)
    am_c1 = gpu_am_c1(vg, barrier)

    serving = run_serving(args) if args.serve_problems > 0 else None

    if rank != 0:
        ctx.close()
        if dist:
            dist.destroy_process_group()
        return

    peaks = _peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    nodes, cells = ctx.N, (n - 1) ** 3
    # algorithmic traffic per apply: read u (24 B) + v (8 B), write y (24 B) per node
    alg_bytes = 56.0 * nodes
    # FP64 instructions per element of the apply on this workload (nearly every element
    # has a constant nodal phase field and takes the fixed-weight element), counted by ncu
    # (smsp__sass_thread_inst_executed_op_{dfma,dadd,dmul}_pred_on / cells, the
    # fixed-weight launch of this workload under ncu --set full); an FMA is 2 flops
    dfma_el, dadd_el, dmul_el = 44.1, 163.7, 25.6
    instr_el = dfma_el + dadd_el + dmul_el
    flops_el = 2 * dfma_el + dadd_el + dmul_el
    f64_peak = fp_peak_tflops(torch, "f64")
    value = N3 * world / (ms64 * 1e-3) / 1e9
    line = {
        "metric": "GDOF/s matvec",
        "value": round(value, 3),
        "unit": "GDOF/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms64, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded random u; v from the penny-crack construction)",
        "config": {"workload": WORKLOAD, "grid": [n, n, n], "u_dofs": N3,
                   "parallelism": f"replicas x{world}", "l2": "flushed between timed steps"},
        "e2e": {"value": round(N3 * world / (e2e_ms * 1e-3) / 1e9, 3), "unit": "GDOF/s",
                "h2d_bytes_per_step": N3 * 8, "d2h_bytes_per_step": N3 * 8},
        "gpu_launches": 3 * args.steps,  # per apply: the two unit-list waves and the seam fix-up
        "roofline": {"bound": "hbm", "achieved": round(alg_bytes / (ms64 * 1e-3) / 1e9, 1),
                     "peak": hbm, "unit": "GB/s",
                     "frac": round(alg_bytes / (ms64 * 1e-3) / 1e9 / hbm, 4),
                     "traffic": 108.7e6 if n == N_EDGE else None,
                     "note": "achieved: algorithmic bytes over the whole apply (three launches: "
                             "the fixed-weight wave over the intact (tile, plane) units, the "
                             "general wave over the rest, the seam fix-up); traffic: ncu dram "
                             "read+write of the fixed-weight launch at 129^3 (84.3 + 24.4 MB; "
                             "part of the output is still in the 126 MB L2 when it ends).  The "
                             "kernel is bound by neither HBM nor the FP64 pipe "
                             "(compute_roofline) but by the latency of its tile schedule "
                             "(ncu: 16 warps per SM, issue active 54 %, FP64 pipe 34 %, top "
                             "stalls fixed-latency dependencies)"},
        "compute_roofline": {
            "pipe": "fp64 CUDA cores",
            "fp64_instructions_per_element": {"dfma": dfma_el, "dadd": dadd_el, "dmul": dmul_el},
            "flops_per_element": round(flops_el, 1),
            "achieved_tflops": round(cells * flops_el / (ms64 * 1e-3) / 1e12, 3),
            "peak_tflops_measured": f64_peak,
            "frac_flops": (round(cells * flops_el / (ms64 * 1e-3) / 1e12 / f64_peak, 3)
                           if f64_peak else None),
            "fp64_pipe_issue_frac": (round(cells * instr_el / (ms64 * 1e-3) / 1e12 / (f64_peak / 2), 3)
                                     if f64_peak else None),
            "note": "frac_flops counts DADD/DMUL as 1 flop; fp64_pipe_issue_frac = FP64 "
                    "instructions issued / (measured DFMA rate), the pipe's occupancy"},
        "mixed": {"value": round(N3 * world / (ms32 * 1e-3) / 1e9, 3), "unit": "GDOF/s",
                  "ms_per_step": round(ms32, 4), "dtype": "f32"},
        "tensor_core_apply": None if not args.tc else {
            "value": round(N3 * world / (mstc * 1e-3) / 1e9, 3), "unit": "GDOF/s",
            "ms_per_step": round(mstc, 4), "dtype": "f32 (split-tf32 tcgen05.mma)",
            "ok": tc_ok,
            "note": "vfgpu_u_apply_tc: element contraction as two GEMMs per 128-element tile on "
                    "the tensor cores (not used by the solvers); compare with `mixed`"},
        "am_steps_per_s": {**{k: round(1.0 / am[k]["s_per_step"], 3) for k in am},
                           "mixed_vs_fp64_max_rel_energy_diff": rel,
                           "mixed_vs_fp64_rel_at_last_step": rel_last,
                           "mixed_vs_fp64_v_linf": v_linf,
                           "vs_fp64_jacobi_max_rel_energy_diff": {
                               k: versus_fp64(k)[0] for k in am if k != "fp64"},
                           "vs_fp64_jacobi_v_linf": {k: versus_fp64(k)[2] for k in am if k != "fp64"},
                           "note": "fp64 / mixed: Jacobi-preconditioned U solve (the reference's); "
                                   "mg_*: multigrid-preconditioned U solve, same stopping test",
                           "steps": args.am_steps,
                           "kspU_last": {k: am[k]["last_kspU"] for k in am},
                           "vs_fp64_oracle": vs_oracle,
                           "c1_41": am_c1},
        "clocks": clocks,
    }
    if serving:
        line["serving"] = serving
    if args.cpu_baseline:
        line["cpu_baseline"] = cpu_reference(args)
    print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()


def versus_oracle(am, vfin, n, its):
    """Each AM variant against the CPU oracle's FP64 run of the same 10 iterations
    (tests/golden/penny129.npz, made by tests/golden/make_penny129.py): the largest
    relative difference of elastic energy, pressure work, surface energy and crack
    opening over the iterations, and the V L-inf difference after the last one."""
    path = os.path.join(ROOT, "tests", "golden", "penny129.npz")
    if n != 129 or its != 10 or not os.path.exists(path):
        return None
    fx = np.load(path)
    rec = fx["rec"][:, :4]
    out = {}
    for key in am:
        e = np.array(am[key]["energies"])
        out[key] = {"max_rel_energy_diff": float((np.abs(e - rec) / np.abs(rec)).max()),
                    "v_linf": float(np.abs(vfin[key] - fx["V"]).max())}
    out["reference"] = "CPU oracle (FP64 restatement of the reference's solves), 10 AM iterations"
    return out


def gpu_am_c1(vg, barrier, its=3):
    """AM steps of the 41^3 penny crack (the CPU AM-step baseline's workload) with the
    Jacobi U solve, FP64 and mixed; the first iteration (from U = 0) untimed."""
    out = {}
    for prec in ("fp64", "mixed"):
        ctx, _ = setup_problem(vg, 41)
        times = []
        for it in range(its):
            barrier()
            t0 = time.perf_counter()
            ctx.am_step(dict(precision=prec))
            barrier()
            times.append(time.perf_counter() - t0)
        ctx.close()
        out[prec] = round(1.0 / float(np.mean(times[1:])), 3)
    out["sample"] = f"AM iterations 2..{its} (the first, from U = 0, untimed)"
    return out


def run_serving(args):
    """The serving stream: independent pressurised-crack problems (grid edge uniform over
    {17, 33, 65, 97}, 1-4 random penny cracks, E ~ U[5,30] GPa, nu ~ U[0.15,0.35], AT1/AT2,
    5 AM iterations each, multigrid U solve on the two larger grids) through the library's
    request loop.  The FP64 capacity is
    measured closed-loop on the whole stream; the stream then arrives as a
    seeded Poisson process at 0.8x that capacity, once in FP64 and once mixed (same
    arrival times).  Latency = completion - arrival."""
    from vpfhf_b200.serve import poisson_arrivals, run_stream, serving_stream
    count, workers = args.serve_problems, args.serve_workers
    # capacity closed-loop on the whole stream: a sample's random mix of grid sizes moved
    # it by +-10 %, and the open-loop latencies at 0.8x with it
    cal = serving_stream(count=count, precision="fp64")
    _, cap = run_stream(cal, None, workers=workers)
    rate = 0.8 * cap["throughput"]
    arr = poisson_arrivals(count, rate)
    out = {"problems": count, "workers": workers, "am_its_per_problem": 5,
           "u_solve": "multigrid PCG on the 65^3 / 97^3 problems, Jacobi PCG on 17^3 / 33^3 "
                      "(solve option pc = auto)",
           "capacity_fp64_per_s": round(cap["throughput"], 3),
           "arrival_rate_per_s": round(rate, 3),
           "grids": "edge uniform over {17,33,65,97}, cube [0,4]^3"}
    keys = ("throughput", "p50_s", "p99_s", "mean_s", "max_s", "failed", "reused",
            "contexts_created", "evictions", "peak_reserved_gb", "span_s")
    for prec in ("fp64", "mixed"):
        _, summ = run_stream(serving_stream(count=count, precision=prec), arr, workers=workers)
        out[prec] = {k: (round(summ[k], 4) if isinstance(summ[k], float) else summ[k])
                     for k in keys}
        out[prec]["throughput_unit"] = "problems/s"
    return out


def _am_run(ctx, prob, prec, its, altmintol=0.0, reset=True, pc="jacobi"):
    """AM iterations on `ctx`: exactly `its` (altmintol 0) or until ||V - Vold||_inf <
    altmintol; returns per-iteration records."""
    import torch
    if reset:
        ctx.set_field("U", np.zeros(3 * ctx.N))
        ctx.init_cracks(prob["pennies"])
        ctx.time_step_prepare()
    recs = []
    for it in range(its):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc, err, su, sv = ctx.am_step(dict(precision=prec, pc=pc))
        dt = time.perf_counter() - t0
        recs.append(dict(s=dt, err=err, rc=rc, kspU=su["ksp_its"], kspV=sv["ksp_its"]))
        if altmintol > 0 and err < altmintol:
            break
    return recs


def c3_run(ctx, prob, prec, pc, args):
    """The quasi-static poroelastic run: pressure scaled k / load_steps for k = 1 ..
    load_steps, each step AM to ||V - Vold||_inf < 1e-3 (at most max_am iterations),
    from U = 0 and the initial cracks.  A progress line per step goes to stderr."""
    ctx.set_field("U", np.zeros(3 * ctx.N))
    ctx.init_cracks(prob["pennies"])
    pfull = prob["pressure"]
    steps, am_total, t_total = [], 0, 0.0
    for k in range(1, min(args.load_steps, args.c3_steps or args.load_steps) + 1):
        ctx.set_field("pressure", pfull * (k / args.load_steps))
        ctx.time_step_prepare()
        recs = _am_run(ctx, prob, prec, args.max_am, altmintol=1e-3, reset=False, pc=pc)
        am_total += len(recs)
        t_total += sum(r["s"] for r in recs)
        steps.append(dict(step=k, am_its=len(recs), last_err=recs[-1]["err"],
                          s=round(sum(r["s"] for r in recs), 3),
                          kspU=[r["kspU"] for r in recs], kspV=[r["kspV"] for r in recs],
                          **_energies(ctx)))
        print(json.dumps({"c3_progress": prec, **steps[-1]}), file=sys.stderr, flush=True)
    return (dict(am_steps=am_total, solve_s=round(t_total, 2),
                 am_steps_per_s=round(am_total / t_total, 4), steps=steps),
            ctx.get_field("V"))


def _energies(ctx):
    el, _, pw = ctx.u_energy()
    return dict(elastic=el, pressure_work=pw, surface=ctx.v_energy(), cov=ctx.crack_opening())


def run_large(args):
    """The large single-GPU set-ups: `c5` (321^3, heterogeneous E, 8 cracks, 10 AM
    iterations, FP64 and mixed from the same start) and `c3` (257x257x129 poroelastic,
    16 cracks, 20 quasi-static pressure steps, AM to 1e-3 or at most --max-am iterations
    per step, FP64 and mixed)."""
    import torch
    import vpfhf_b200 as vg
    from vpfhf_b200 import workloads as wl
    rank, world, local = _rank()
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    make = wl.c5_problem if args.config == "c5" else wl.c3_problem
    full = (321, 321, 321) if args.config == "c5" else (257, 257, 129)
    # --scale < 1: a smaller instance of the same set-up (probes); cells scale linearly
    n = tuple(max(9, int(round((k - 1) * args.scale)) + 1) for k in full)
    prob = make(n=n)
    gen_s = time.perf_counter() - t0
    ctx = wl.make_context(vg, prob)
    n = prob["n"]
    out = {"config": args.config, "grid": list(n), "u_dofs": 3 * ctx.N, "setup_s": round(gen_s, 2),
           "cracks": len(prob["pennies"])}
    if args.config == "c5":
        res, fields = {}, {}
        variants = [v for v in AM_VARIANTS if args.pc == "both" or v[2] == args.pc]
        if variants[0][0] != "fp64":  # the FP64 Jacobi run is the reference for the diffs
            variants.insert(0, AM_VARIANTS[0])
        for key, prec, pc in variants:
            recs = _am_run(ctx, prob, prec, args.am_steps, pc=pc)
            res[key] = dict(s_per_step=float(np.mean([r["s"] for r in recs[1:]])),
                            kspU=[r["kspU"] for r in recs], kspV=[r["kspV"] for r in recs],
                            **_energies(ctx))
            fields[key] = ctx.get_field("V")
        ekeys = ("elastic", "pressure_work", "surface", "cov")
        out.update({
            "am_its": args.am_steps,
            "am_steps_per_s": {k: round(1.0 / res[k]["s_per_step"], 4) for k in res},
            "over_fp64": {k: round(res["fp64"]["s_per_step"] / res[k]["s_per_step"], 3)
                          for k in res if k != "fp64"},
            "vs_fp64_rel": {k: {e: abs(res[k][e] - res["fp64"][e]) / abs(res["fp64"][e])
                                for e in ekeys} for k in res if k != "fp64"},
            "vs_fp64_v_linf": {k: float(np.abs(fields[k] - fields["fp64"]).max())
                               for k in res if k != "fp64"},
            **res})
    else:
        pc = "mg" if args.pc == "both" else args.pc
        runs, fields = {}, {}
        for prec in ("fp64", "mixed"):
            runs[prec], fields[prec] = c3_run(ctx, prob, prec, pc, args)
        ekeys = ("elastic", "pressure_work", "surface", "cov")
        last = {p: runs[p]["steps"][-1] for p in runs}
        out.update({"pc": pc, "load_steps": args.load_steps,
                    "steps_run": len(runs["fp64"]["steps"]), "altmintol": 1e-3,
                    "max_am_per_step": args.max_am,
                    "am_steps_per_s": {p: runs[p]["am_steps_per_s"] for p in runs},
                    "mixed_vs_fp64_rel_at_last_step": {  # absolute where the FP64 value is 0
                        e: abs(last["mixed"][e] - last["fp64"][e]) / (abs(last["fp64"][e]) or 1.0)
                        for e in ekeys},
                    "mixed_vs_fp64_v_linf": float(np.abs(fields["mixed"] - fields["fp64"]).max()),
                    **runs})
    ctx.close()
    if rank == 0:
        print(json.dumps(out))


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_reference(args, reps=5):
    """The reference's method on the host cores, restated in the oracle (oracle/):
    the KSP matvec -- the assembled DMDA AIJ matrix (CSR, 81 nnz/row) times a vector --
    on the 129^3 workload itself, and the AM step (StepU + StepV with re-formed element
    matrices, the Jacobian assembled every Newton iteration and CG + Jacobi on the
    assembled matrix) on the 41^3 penny crack."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import vforacle as vo
    n = N_EDGE
    h = L_BOX / (n - 1)
    cores = os.cpu_count() or 1
    o = vo.Oracle((n, n, n), (L_BOX,) * 3, E=1e10, nu=0.25, Gc=100.0, epsilon=2 * h, eta=1e-8,
                  atnum=1, nthreads=cores)
    v = o.penny_v((L_BOX / 2,) * 3, 0.4)
    mask, _ = o.bc(vo.rollers_face())
    t0 = time.perf_counter()
    csr = o.u_csr(v, mask)
    t_asm = time.perf_counter() - t0
    x = np.random.default_rng(7).standard_normal(3 * o.N)
    o.csr_spmv(csr, x, cores)
    t0 = time.perf_counter()
    for _ in range(reps):
        o.csr_spmv(csr, x, cores)
    dt = (time.perf_counter() - t0) / reps
    nnz = len(csr[1])
    del csr
    am = cpu_am_step(vo, cores)
    return {"value": round(3 * o.N / dt / 1e9, 4), "unit": "GDOF/s", "cores": cores,
            "kind": "port", "cpu": _cpu_model(),
            "sample": f"AIJ (CSR, 81 nnz/row) SpMV of K(v) on the 129^3 penny-crack grid "
                      f"({3 * o.N} dofs, {nnz} nonzeros), {reps} products after one untimed",
            "assembly_s": round(t_asm, 3),
            "am_step": am}


def cpu_am_step(vo, cores, its=3):
    """AM iterations of the 41^3 pressurised penny crack (E 10 GPa, nu 0.25, Gc 100, AT1,
    eps 2h, p 1 MPa, rollers) by the reference's method on all host cores; the first
    iteration (from U = 0) is untimed, the rest averaged."""
    n, h = 41, L_BOX / 40
    o = vo.Oracle((n, n, n), (L_BOX,) * 3, E=1e10, nu=0.25, Gc=100.0, epsilon=2 * h, eta=1e-8,
                  atnum=1, nthreads=cores)
    V = o.penny_v((L_BOX / 2,) * 3, 0.4)
    virrev = V.copy()
    U = np.zeros(3 * o.N)
    p = np.full(o.N, 1e6)
    umask, uval = o.bc(vo.rollers_face())
    lb, ub = np.zeros(o.N), virrev.copy()
    recs = []
    for it in range(its):
        t0 = time.perf_counter()
        su, ta_u = o.step_u_asm(U, V, p=p, mask=umask, value=uval)
        t1 = time.perf_counter()
        sv, ta_v = o.step_v_asm(V, U, lb, ub, p=p)
        t2 = time.perf_counter()
        recs.append(dict(s=t2 - t0, u_s=t1 - t0, v_s=t2 - t1, asm_s=ta_u + ta_v,
                         kspU=su.ksp_its, kspV=sv.ksp_its))
    timed = recs[1:]
    s = float(np.mean([r["s"] for r in timed]))
    return {"workload": "penny crack 41^3 (206,763 U dofs), AT1 eps=2h, rollers, p=1e6",
            "method": "assembled Jacobians (CSR) + CG/Jacobi, residuals from element matrices",
            "am_steps_per_s": round(1.0 / s, 4), "s_per_step": round(s, 3),
            "assembly_share": round(float(np.mean([r["asm_s"] / r["s"] for r in timed])), 3),
            "kspU": [r["kspU"] for r in recs], "kspV": [r["kspV"] for r in recs],
            "sample": f"AM iterations 2..{its} (the first, from U = 0, untimed)"}


def run_reference(args):
    rank, world, _ = _rank()
    if rank != 0:
        return
    cb = cpu_reference(args)
    print(json.dumps({
        "impl": "reference", "metric": "GDOF/s matvec", "value": cb["value"], "unit": "GDOF/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": [N_EDGE] * 3, "sample": cb["sample"]},
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": "GDOF/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--am-steps", type=int, default=10)
    ap.add_argument("--serve-problems", type=int, default=512,
                    help="problems in the serving stream (0 skips it)")
    ap.add_argument("--serve-workers", type=int, default=8)
    ap.add_argument("--impl", default="vfgpu", choices=["vfgpu", "reference"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-tc", dest="tc", action="store_false",
                    help="skip the tensor-core apply timing")
    ap.add_argument("--grid", type=int, default=N_EDGE, help="nodes per axis (profiling runs)")
    ap.add_argument("--only-apply", action="store_true",
                    help="time the operator applications only (profiling runs)")
    ap.add_argument("--config", default="c2", choices=["c2", "c3", "c5"],
                    help="c2: the headline line; c3 / c5: the large set-ups (one JSON line)")
    ap.add_argument("--load-steps", type=int, default=20, help="c3 quasi-static steps")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="c3 / c5: cells per axis scaled by this factor (1 = the full set-up)")
    ap.add_argument("--max-am", type=int, default=5, help="c3 AM cap per load step")
    ap.add_argument("--c3-steps", type=int, default=0,
                    help="c3: run only the first this many of the --load-steps steps (0 = all)")
    ap.add_argument("--pc", default="both", choices=["jacobi", "mg", "both"],
                    help="U preconditioner of the c3 / c5 runs (c3: both = mg)")
    ap.add_argument("--only-am", action="store_true",
                    help="run the AM steps only, with a per-solve breakdown; the last step of "
                         "--profile-precision is bracketed by cudaProfilerStart/Stop")
    ap.add_argument("--profile-precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--am-pc", default="jacobi", choices=["jacobi", "mg"],
                    help="U preconditioner of the --only-am runs")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.config in ("c3", "c5"):
        run_large(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
