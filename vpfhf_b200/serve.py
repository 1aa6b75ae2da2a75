"""Serving: independent fracture problems through the library's request loop
(vfgpu_server_* in include/vfgpu.h).

The loop itself is native (worker threads, memory-based admission, pooled
contexts with their captured CUDA graphs); this module builds requests, drives
an open-loop arrival process and summarises latencies.  No counterpart in the
reference, which solves one problem per process.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from . import BCSpec, penny_array, rect_array, rollers, solve_opts


@dataclass
class Problem:
    """One fracture problem: grid, one material, phase-field parameters, cracks and
    a uniform crack pressure on rollers (the pressurised-crack set-up of the
    reference's test18 / VPFHF runs), solved by `am_its` AM iterations."""
    n: tuple = (17, 17, 17)
    l: tuple = (4.0, 4.0, 4.0)
    E: float = 1e10
    nu: float = 0.25
    Gc: float = 100.0
    alpha: float = 0.0
    beta: float = 0.0
    epsilon: float | None = None  # None: 2 h (h the x spacing)
    eta: float = 1e-8
    irrevtol: float = 5e-2
    atnum: int = 1
    pressure: float = 1e6
    pressurize: bool = True
    pennies: list = field(default_factory=list)  # dicts (center, r, theta, phi, thickness)
    rects: list = field(default_factory=list)    # dicts (corners, thickness)
    am_its: int = 5
    altmintol: float = 0.0
    max_am_its: int = 0
    precision: str = "fp64"
    pc: str = "jacobi"  # StepU preconditioner: "jacobi" (the reference's) or "mg"
    bcU: list | None = None  # three BCSpec (default rollers)
    bcV: BCSpec | None = None
    tag: int = 0

    @property
    def eps(self):
        return self.epsilon if self.epsilon is not None else 2.0 * self.l[0] / (self.n[0] - 1)

    @property
    def nodes(self):
        return self.n[0] * self.n[1] * self.n[2]


def make_request(p: Problem, out_u=None, out_v=None, out_cellcov=None) -> _abi.Request:
    q = _abi.Request()
    q.grid = _abi.Grid(*(int(v) for v in p.n), *(float(v) for v in p.l))
    q.mp = _abi.MatProp(p.E, p.nu, p.alpha, p.beta, p.Gc)
    q.vf = _abi.VFProp(p.eps, p.eta, p.irrevtol, int(p.atnum), int(bool(p.pressurize)))
    for c, b in enumerate(p.bcU or rollers()):
        q.bcU[c] = b.to_c()
    q.bcV = (p.bcV or BCSpec()).to_c()
    q.pressure = p.pressure
    if len(p.pennies) > _abi.SERVE_MAX_PENNY or len(p.rects) > _abi.SERVE_MAX_RECT:
        raise ValueError("too many cracks for one request")
    pa, ra = penny_array(p.pennies), rect_array(p.rects)
    q.npenny, q.nrect = len(pa), len(ra)
    for i in range(len(pa)):
        q.penny[i] = pa[i]
    for i in range(len(ra)):
        q.rect[i] = ra[i]
    q.am_its, q.altmintol, q.max_am_its = p.am_its, p.altmintol, p.max_am_its
    q.opts = solve_opts(precision=p.precision, pc=p.pc)
    q.out_u = _abi.ptr(out_u)
    q.out_v = _abi.ptr(out_v)
    q.out_cellcov = _abi.ptr(out_cellcov)
    q.tag = p.tag
    return q


class Server:
    """vfgpu_server: `workers` threads on the current CUDA device; budget_bytes <= 0
    means 85 % of the free device memory."""

    def __init__(self, workers=8, budget_bytes=0, device=None):
        self.L = _abi.lib()
        if device is None:
            import torch
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        h = C.c_void_p()
        _abi.check(self.L.vfgpu_server_create(int(device), int(workers), int(budget_bytes),
                                              C.byref(h)), "vfgpu_server_create")
        self.h = h
        self._keep = {}  # ticket -> output arrays the server writes into
        self._lock = threading.Lock()

    def submit(self, p: Problem, out_u=None, out_v=None, out_cellcov=None) -> int:
        q = make_request(p, out_u, out_v, out_cellcov)
        t = C.c_ulonglong()
        with self._lock:
            _abi.check(self.L.vfgpu_server_submit(self.h, C.byref(q), C.byref(t)),
                       "vfgpu_server_submit")
            self._keep[t.value] = (out_u, out_v, out_cellcov)
        return t.value

    def next(self, timeout=-1.0):
        """The next finished problem's result (dict), or None after `timeout` seconds."""
        r = _abi.Result()
        rc = _abi.check(self.L.vfgpu_server_next(self.h, float(timeout), C.byref(r)),
                        "vfgpu_server_next")
        if rc != _abi.OK:
            return None
        with self._lock:
            self._keep.pop(r.ticket, None)
        return r.as_dict()

    def clock(self):
        return self.L.vfgpu_server_clock(self.h)

    def info(self):
        i = _abi.ServerInfo()
        _abi.check(self.L.vfgpu_server_info_get(self.h, C.byref(i)), "vfgpu_server_info_get")
        return i.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.L.vfgpu_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# -- the serving workload: random pressurised-crack problems -------------------------
def random_penny(rng, L):
    """A penny crack with a normal uniform on the sphere, radius U[0.05, 0.2] L and the
    center uniform in the inner 60 % of the box."""
    theta = rng.uniform(0.0, 360.0)
    phi = math.degrees(math.acos(1.0 - 2.0 * rng.uniform()))
    r = rng.uniform(0.05, 0.2) * L[0]
    center = [rng.uniform(0.2 * x, 0.8 * x) for x in L]
    return dict(center=center, r=r, theta=theta, phi=phi, thickness=0.0)


def serving_stream(count=512, seed=1004, edges=(17, 33, 65, 97), L=4.0, am_its=5,
                   precision="fp64", pc="auto"):
    """`count` independent problems: grid edge uniform over `edges`, 1-4 random penny
    cracks, E ~ U[5, 30] GPa, nu ~ U[0.15, 0.35], AT1 or AT2 with probability 1/2,
    epsilon = 2h, eta = 1e-8, Gc = 100, 1 MPa crack pressure on rollers.  `pc` "auto"
    solves the 65^3 and 97^3 problems with the multigrid U solve and the smaller ones
    with the Jacobi one."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        e = int(edges[rng.integers(len(edges))])
        box = (L, L, L)
        ncr = int(rng.integers(1, 5))
        pennies = [random_penny(rng, box) for _ in range(ncr)]
        out.append(Problem(n=(e, e, e), l=box, E=rng.uniform(5e9, 30e9),
                           nu=rng.uniform(0.15, 0.35), atnum=1 if rng.uniform() < 0.5 else 2,
                           pennies=pennies, am_its=am_its, precision=precision, pc=pc,
                           tag=i))
    return out


def poisson_arrivals(count, rate, seed=1004):
    """Arrival times (s) of a Poisson process of `rate` per second."""
    rng = np.random.default_rng(seed + 7919)
    return np.cumsum(rng.exponential(1.0 / rate, count))


def run_stream(problems, arrivals=None, workers=8, budget_bytes=0, server=None):
    """Submits problems[i] at arrivals[i] seconds after the start (all at once if
    arrivals is None), collects every result and returns (results by tag, summary).
    Latency = completion - submission, both on the server clock."""
    own = server is None
    srv = server or Server(workers=workers, budget_bytes=budget_bytes)
    results = {}
    done = threading.Event()

    def collect():
        for _ in range(len(problems)):
            r = srv.next(-1.0)
            results[r["tag"]] = r
        done.set()

    th = threading.Thread(target=collect, daemon=True)
    th.start()
    t0 = srv.clock()
    for i, p in enumerate(problems):
        if arrivals is not None:
            wait = t0 + arrivals[i] - srv.clock()
            if wait > 0:
                time.sleep(wait)
        srv.submit(p)
    done.wait()
    th.join()
    info = srv.info()
    if own:
        srv.close()
    lat = np.array([r["t_done"] - r["t_submit"] for r in results.values()])
    first = min(r["t_submit"] for r in results.values())
    last = max(r["t_done"] for r in results.values())
    bad = [r for r in results.values() if r["status"] < 0]
    summary = dict(problems=len(problems), failed=len(bad), span_s=last - first,
                   throughput=len(problems) / (last - first),
                   p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
                   mean_s=float(lat.mean()), max_s=float(lat.max()),
                   am_steps=int(sum(r["am_its"] for r in results.values())),
                   reused=int(sum(r["reused_ctx"] for r in results.values())),
                   contexts_created=info["contexts_created"], evictions=info["evictions"],
                   peak_reserved_gb=info["peak_reserved_bytes"] / 1e9, workers=info["workers"])
    if bad:
        summary["first_error"] = bad[0]["error"]
    return results, summary
