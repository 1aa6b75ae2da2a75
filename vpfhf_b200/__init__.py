"""vpfhf_b200 -- B200 (sm_100a) implementation of VPFHF's alternate-minimisation
hot path: the phase-field-degraded Q1-hex displacement operator (U), the
AT1/AT2 damage operator (V), their solves and energies.

The compute runs in libvfgpu.so (CUDA, behind the C ABI in include/vfgpu.h);
this module is the host-side mirror of the reference's interface
(VFCtx/VFFields + VF_StepU, VF_StepV, VF_UEnergy3D, VF_VEnergy3D,
VolumetricCrackOpening) over that ABI.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import (BC_FIXED, BC_NONE, BC_ONE, BC_ZERO, FP64, MIXED, VFGPUError)  # noqa: F401

__all__ = ["VFContext", "BCSpec", "rollers", "solve_opts", "bc_vector", "FP64", "MIXED",
           "VFGPUError", "VF_StepU", "VF_StepV", "VF_UEnergy3D", "VF_VEnergy3D",
           "VolumetricCrackOpening", "VFTimeStepPrepare"]


class BCSpec:
    """One VFBC (VFCartFE.h:137-144): face[6] / vertex[8] BC types and values."""

    FACES = ("X0", "X1", "Y0", "Y1", "Z0", "Z1")
    VERTICES = ("X0Y0Z0", "X1Y0Z0", "X0Y1Z0", "X1Y1Z0", "X0Y0Z1", "X1Y0Z1", "X0Y1Z1", "X1Y1Z1")

    def __init__(self, **kw):
        self.face = [BC_NONE] * 6
        self.faceValue = [0.0] * 6
        self.vertex = [BC_NONE] * 8
        self.vertexValue = [0.0] * 8
        for k, t in kw.items():
            val = 0.0
            if isinstance(t, tuple):
                t, val = t
            if k in self.FACES:
                self.face[self.FACES.index(k)] = t
                self.faceValue[self.FACES.index(k)] = val
            elif k in self.VERTICES:
                self.vertex[self.VERTICES.index(k)] = t
                self.vertexValue[self.VERTICES.index(k)] = val
            else:
                raise KeyError(k)

    def to_c(self):
        b = _abi.BC()
        for i in range(6):
            b.face[i], b.faceValue[i] = self.face[i], self.faceValue[i]
        for i in range(8):
            b.vertex[i], b.vertexValue[i] = self.vertex[i], self.vertexValue[i]
        return b


def rollers():
    """BCfiles/3DRollers.txt: the normal displacement is ZERO on every face."""
    return [BCSpec(X0=BC_ZERO, X1=BC_ZERO), BCSpec(Y0=BC_ZERO, Y1=BC_ZERO),
            BCSpec(Z0=BC_ZERO, Z1=BC_ZERO)]


class VFContext:
    """A problem resident on the current CUDA device (VFCtx + VFFields)."""

    def __init__(self, n, l, matprop, epsilon=0.2, eta=1e-5, irrevtol=5e-2, atnum=2,
                 pressurize=False, layer=None):
        self.L = _abi.lib()
        nx, ny, nz = (int(v) for v in n)
        self.n = (nx, ny, nz)
        self.N = nx * ny * nz
        g = _abi.Grid(nx, ny, nz, *(float(v) for v in l))
        h = C.c_void_p()
        _abi.check(self.L.vfgpu_create(C.byref(g), C.byref(h)), "vfgpu_create")
        self.h = h
        self.set_matprop(matprop, layer)
        self.set_vfprop(epsilon, eta, irrevtol, atnum, pressurize)

    def close(self):
        if getattr(self, "h", None):
            self.L.vfgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- set-up ---------------------------------------------------------------
    def set_matprop(self, matprop, layer=None):
        """matprop: dict or list of dicts with E, nu, alpha, beta, Gc (per layer)."""
        if isinstance(matprop, dict):
            matprop = [matprop]
        arr = (_abi.MatProp * len(matprop))()
        for i, m in enumerate(matprop):
            arr[i] = _abi.MatProp(m.get("E", 1.0), m.get("nu", 0.0), m.get("alpha", 0.0),
                                  m.get("beta", 0.0), m.get("Gc", 1.0))
        lay = None
        if layer is not None:
            lay = np.ascontiguousarray(layer, dtype=np.int32)
        _abi.check(self.L.vfgpu_set_matprop(self.h, len(matprop), arr, _abi.ptr(lay)),
                   "vfgpu_set_matprop")

    def set_cell_modulus(self, cellE):
        arr = None if cellE is None else np.ascontiguousarray(cellE, dtype=np.float64)
        _abi.check(self.L.vfgpu_set_cell_modulus(self.h, _abi.ptr(arr)), "vfgpu_set_cell_modulus")

    def set_vfprop(self, epsilon, eta, irrevtol=5e-2, atnum=2, pressurize=False):
        vf = _abi.VFProp(float(epsilon), float(eta), float(irrevtol), int(atnum),
                         int(bool(pressurize)))
        _abi.check(self.L.vfgpu_set_vfprop(self.h, C.byref(vf)), "vfgpu_set_vfprop")

    def set_unilateral(self, kind):
        """-unilateral: 0 / "none" or 1 / "nocompression"."""
        if isinstance(kind, str):
            kind = {"none": 0, "nocompression": 1}[kind.lower()]
        _abi.check(self.L.vfgpu_set_unilateral(self.h, int(kind)), "vfgpu_set_unilateral")

    def set_u_split(self, mode):
        """How U applies split their work: "auto" (default), "off" (one wave) or "on"
        (fixed-weight wave over the intact units, general wave over the rest)."""
        if isinstance(mode, str):
            mode = {"auto": 0, "off": 1, "on": 2}[mode.lower()]
        _abi.check(self.L.vfgpu_set_u_split(self.h, int(mode)), "vfgpu_set_u_split")

    def set_insitu(self, smin, smax=None):
        """In-situ stresses (Voigt s11 s22 s33 s23 s13 s12) at z = 0 and z = lz
        (-insitumin / -insitumax); None switches them off."""
        a = None if smin is None else np.ascontiguousarray(smin, dtype=np.float64)
        b = None if smax is None else np.ascontiguousarray(smax, dtype=np.float64)
        _abi.check(self.L.vfgpu_set_insitu(self.h, _abi.ptr(a), _abi.ptr(b)), "vfgpu_set_insitu")

    def set_bc(self, bcU, bcV=None):
        u = (_abi.BC * 3)(*[b.to_c() for b in bcU])
        v = (bcV or BCSpec()).to_c()
        _abi.check(self.L.vfgpu_set_bc(self.h, u, C.byref(v)), "vfgpu_set_bc")

    # -- fields ---------------------------------------------------------------
    def _flen(self, name):
        return 3 * self.N if name in ("U", "BCU") else self.N

    def set_field(self, name, data):
        if isinstance(data, np.ndarray):
            data = np.ascontiguousarray(data, dtype=np.float64)
            assert data.size == self._flen(name), (name, data.size)
        _abi.check(self.L.vfgpu_set_field(self.h, _abi.FIELD_NAMES[name], _abi.ptr(data)),
                   "vfgpu_set_field")

    def get_field(self, name, out=None):
        if out is None:
            out = np.empty(self._flen(name))
        _abi.check(self.L.vfgpu_get_field(self.h, _abi.FIELD_NAMES[name], _abi.ptr(out)),
                   "vfgpu_get_field")
        return out

    # -- operators --------------------------------------------------------------
    def u_apply(self, x, precision=FP64, out=None):
        """y = J_U x with the resident V (VF_UIJacobian applied matrix-free)."""
        if isinstance(x, np.ndarray):
            x = np.ascontiguousarray(x, dtype=np.float64)
        if out is None:
            out = np.empty(3 * self.N) if isinstance(x, np.ndarray) else x.new_empty(3 * self.N)
        _abi.check(self.L.vfgpu_u_apply(self.h, int(precision), _abi.ptr(x), _abi.ptr(out)),
                   "vfgpu_u_apply")
        return out

    def u_apply_dev(self, x, y, precision=FP64):
        """Queues y = J_U x on the ctx stream; x, y are device tensors (float64 for FP64,
        float32 for MIXED).  Returns immediately."""
        _abi.check(self.L.vfgpu_u_apply_dev(self.h, int(precision), x.data_ptr(), y.data_ptr()),
                   "vfgpu_u_apply_dev")

    def u_apply_tc(self, x, y):
        """Queues y = J_U x with the tensor-core element contraction (float32 device
        tensors; vfgpu_u_apply_tc).  Returns immediately."""
        _abi.check(self.L.vfgpu_u_apply_tc(self.h, x.data_ptr(), y.data_ptr()), "vfgpu_u_apply_tc")

    def tc_error(self):
        f = C.c_int()
        _abi.check(self.L.vfgpu_tc_error(self.h, C.byref(f)), "vfgpu_tc_error")
        return bool(f.value)

    @property
    def stream_handle(self):
        s = C.c_void_p()
        _abi.check(self.L.vfgpu_get_stream(self.h, C.byref(s)), "vfgpu_get_stream")
        return s.value

    def torch_stream(self):
        """The ctx stream as a torch.cuda.ExternalStream (for events / ordering)."""
        import torch
        return torch.cuda.ExternalStream(self.stream_handle)

    def init_cracks(self, pennies=(), rects=()):
        """Device crack initialisation (VFFieldsInitialize, VFCommon.c:823-857): V = VIrrev =
        min over the cracks.  pennies: dicts (center, r, theta, phi, thickness) or rows
        (cx, cy, cz, r, theta, phi, thickness); rects: dicts (corners, thickness) or rows
        (9 corners, thickness)."""
        pa, ra = penny_array(pennies), rect_array(rects)
        _abi.check(self.L.vfgpu_init_cracks(self.h, len(pa), pa if len(pa) else None, len(ra),
                                            ra if len(ra) else None), "vfgpu_init_cracks")

    # -- solves ---------------------------------------------------------------------
    def step_u(self, opts=None):
        """VF_StepU: returns (status, stats dict); status 0 converged, 1 not converged,
        2 diverged."""
        st = _abi.SolveStats()
        o = solve_opts(**(opts or {}))
        rc = _abi.check(self.L.vfgpu_step_u(self.h, C.byref(o), C.byref(st)), "vfgpu_step_u")
        return rc, st.as_dict()

    def step_v(self, opts=None):
        """VF_StepV (VI Newton with bounds [0,1] or [0,VIrrev])."""
        st = _abi.SolveStats()
        o = solve_opts(**(opts or {}))
        rc = _abi.check(self.L.vfgpu_step_v(self.h, C.byref(o), C.byref(st)), "vfgpu_step_v")
        return rc, st.as_dict()

    def am_step(self, opts=None):
        """StepU + StepV; returns (status, errV, statsU, statsV)."""
        su, sv, err = _abi.SolveStats(), _abi.SolveStats(), C.c_double()
        o = solve_opts(**(opts or {}))
        rc = _abi.check(self.L.vfgpu_am_step(self.h, C.byref(o), C.byref(err), C.byref(su),
                                             C.byref(sv)), "vfgpu_am_step")
        return rc, err.value, su.as_dict(), sv.as_dict()

    def time_step_prepare(self):
        _abi.check(self.L.vfgpu_time_step_prepare(self.h), "vfgpu_time_step_prepare")

    def u_energy(self):
        """(elastic energy, in-situ work, pressure work) as VF_UEnergy3D."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _abi.check(self.L.vfgpu_u_energy(self.h, C.byref(a), C.byref(b), C.byref(c)),
                   "vfgpu_u_energy")
        return a.value, b.value, c.value

    def v_energy(self):
        s = C.c_double()
        _abi.check(self.L.vfgpu_v_energy(self.h, C.byref(s)), "vfgpu_v_energy")
        return s.value

    def update_fracture_width(self, int_length=0.0, width_tol=0.1, remove_tip_effect=False):
        """UpdateFractureWidth (VFPermfield.c:267-562) at the resident U and V: returns
        (widthc per cell, width per node, pmult per cell, stalled band cells).
        int_length <= 0 takes WidthIntLenght = 3 res + 4 epsilon (VFCommon.c:897-914)."""
        o = _abi.WidthOpts(float(int_length), float(width_tol), int(bool(remove_tip_effect)))
        n = self.n
        nc = (n[0] - 1) * (n[1] - 1) * (n[2] - 1)
        wc, wn, pm, st = np.empty(nc), np.empty(self.N), np.empty(nc), C.c_int()
        _abi.check(self.L.vfgpu_update_fracture_width(self.h, C.byref(o), _abi.ptr(wc),
                                                      _abi.ptr(wn), _abi.ptr(pm), C.byref(st)),
                   "vfgpu_update_fracture_width")
        return wc, wn, pm, st.value

    def cell_to_node(self, cellv):
        """CellToNodeInterpolation (VFPermfield.c:1156-1330) of a scalar cell field."""
        cv = np.ascontiguousarray(cellv, np.float64)
        out = np.empty(self.N)
        _abi.check(self.L.vfgpu_cell_to_node(self.h, _abi.ptr(cv), _abi.ptr(out)),
                   "vfgpu_cell_to_node")
        return out

    def fracture_well_rate(self, regrate):
        """VolumetricFractureWellRate (VFPermfield.c:1552-1604) of a nodal rate field."""
        r = C.c_double()
        reg = np.ascontiguousarray(regrate, np.float64)
        _abi.check(self.L.vfgpu_fracture_well_rate(self.h, _abi.ptr(reg), C.byref(r)),
                   "vfgpu_fracture_well_rate")
        return r.value

    def crack_opening(self, cell=False):
        cov = C.c_double()
        n = self.n
        cc = np.empty((n[0] - 1) * (n[1] - 1) * (n[2] - 1)) if cell else None
        _abi.check(self.L.vfgpu_crack_opening(self.h, C.byref(cov), _abi.ptr(cc)),
                   "vfgpu_crack_opening")
        return (cov.value, cc) if cell else cov.value

    def u_residual(self):
        F = np.empty(3 * self.N)
        _abi.check(self.L.vfgpu_u_residual(self.h, _abi.ptr(F)), "vfgpu_u_residual")
        return F

    def v_residual(self):
        F = np.empty(self.N)
        _abi.check(self.L.vfgpu_v_residual(self.h, _abi.ptr(F)), "vfgpu_v_residual")
        return F


def solve_opts(**kw):
    """SolveOpts with the reference's defaults (vfgpu_default_solve_opts), overridden by kw;
    `precision` accepts FP64 / MIXED or "fp64" / "mixed", `pc` "jacobi" / "mg" / "auto"
    (multigrid on grids with >= 65 nodes along some axis, else Jacobi)."""
    o = _abi.SolveOpts()
    _abi.lib().vfgpu_default_solve_opts(C.byref(o))
    for k, v in kw.items():
        if k == "precision" and isinstance(v, str):
            v = {"fp64": FP64, "mixed": MIXED}[v.lower()]
        if k == "pc" and isinstance(v, str):
            v = {"jacobi": _abi.PC_JACOBI, "mg": _abi.PC_MG, "auto": _abi.PC_AUTO}[v.lower()]
        setattr(o, k, v)
    return o


def mg_hierarchy(shape, lengths=(1.0, 1.0, 1.0), precision=MIXED):
    """The multigrid levels (node counts per axis) a pc="mg" solve builds for this grid,
    and the hierarchy's extra device bytes for the V-cycle precision (FP32 under MIXED,
    FP64 under FP64).  Host only.  One level: the grid cannot be coarsened."""
    g = _abi.Grid(*shape, *lengths)
    dims = (C.c_int * 96)()
    nlev, nbytes = C.c_int(0), C.c_longlong(0)
    _abi.check(_abi.lib().vfgpu_mg_hierarchy(C.byref(g), 4 if precision == MIXED else 8, 32, dims,
                                               C.byref(nlev), C.byref(nbytes)),
               "vfgpu_mg_hierarchy")
    return [tuple(dims[3 * l:3 * l + 3]) for l in range(min(nlev.value, 32))], nbytes.value


def penny_crack_v(n, l, center, r, theta=0.0, phi=0.0, thickness=0.0, epsilon=0.2, atnum=1):
    """Initial phase field of one penny-shaped crack, VFPennyCrackBuildVAT1/2
    (VFCracks.c:136-227) with the distance of VFDistanceToPennyCrack (VFCracks.c:101-126):
    disk normal (cos th sin ph, sin th sin ph, cos ph) in degrees; v = 0 within
    thickness/2 of the disk; AT1 profile d/eps (1 - d/(4 eps)) for d < 2 eps, AT2
    1 - exp(-d/(2 eps)).  Several cracks combine by pointwise minimum
    (VFFieldsInitialize, VFCommon.c:829-857)."""
    nx, ny, nz = n
    x = [np.arange(k) * (L / (k - 1)) for k, L in zip(n, l)]
    Z, Y, X = np.meshgrid(x[2], x[1], x[0], indexing="ij")
    t, p = np.deg2rad(theta), np.deg2rad(phi)
    nrm = (np.cos(t) * np.sin(p), np.sin(t) * np.sin(p), np.cos(p))
    dx, dy, dz = X - center[0], Y - center[1], Z - center[2]
    xn = dx * nrm[0] + dy * nrm[1] + dz * nrm[2]
    tx, ty, tz = dx - xn * nrm[0], dy - xn * nrm[1], dz - xn * nrm[2]
    lt = np.sqrt(tx * tx + ty * ty + tz * tz)
    d = np.where(lt <= r, np.abs(xn), np.sqrt(xn ** 2 + (lt - r) ** 2)) - thickness / 2.0
    if r == 0:
        return np.ones(nx * ny * nz)
    if atnum == 1:
        v = np.where(d <= 0, 0.0, np.where(d < 2 * epsilon, d / epsilon * (1 - 0.25 * d / epsilon),
                                          1.0))
    else:
        v = np.where(d <= 0, 0.0, 1.0 - np.exp(-np.maximum(d, 0) / 2 / epsilon))
    return np.ascontiguousarray(v).reshape(-1)


def _penny(p):
    if isinstance(p, dict):
        return _abi.Penny((C.c_double * 3)(*p["center"]), p["r"], p.get("theta", 0.0),
                          p.get("phi", 0.0), p.get("thickness", 0.0))
    return _abi.Penny((C.c_double * 3)(*p[:3]), *p[3:7])


def _rect(r):
    if isinstance(r, dict):
        return _abi.Rect((C.c_double * 9)(*r["corners"]), r.get("thickness", 0.0))
    return _abi.Rect((C.c_double * 9)(*r[:9]), r[9])


def penny_array(pennies):
    return (_abi.Penny * len(pennies))(*[_penny(p) for p in pennies])


def rect_array(rects):
    return (_abi.Rect * len(rects))(*[_rect(r) for r in rects])


def bc_vector(n, bcs):
    """VecSetFromBC (VFCartFE.c:279-491): the vector of Dirichlet values of a VFBC array
    (face values in face order X0,X1,Y0,Y1,Z0,Z1, then vertex values); dof = len(bcs)."""
    nx, ny, nz = n
    dof = len(bcs)
    out = np.zeros((nz, ny, nx, dof))
    for c, b in enumerate(bcs):
        for f in range(6):
            t = b.face[f]
            if t == BC_NONE:
                continue
            val = 0.0 if t == BC_ZERO else 1.0 if t == BC_ONE else b.faceValue[f]
            sl = [slice(None)] * 3
            axis = 2 - f // 2          # X -> last array axis
            sl[axis] = 0 if f % 2 == 0 else n[f // 2] - 1
            out[tuple(sl) + (c,)] = val
        for o in (0, 4, 2, 6, 1, 5, 3, 7):
            t = b.vertex[o]
            if t == BC_NONE:
                continue
            val = 0.0 if t == BC_ZERO else 1.0 if t == BC_ONE else b.vertexValue[o]
            i = nx - 1 if o & 1 else 0
            j = ny - 1 if o & 2 else 0
            k = nz - 1 if o & 4 else 0
            out[k, j, i, c] = val
    return out.reshape(-1)


# -- the reference's entry points over a VFContext ---------------------------------
def VF_StepU(ctx, opts=None):
    """VF_StepU (VFMech.c:1436): returns the SNES converged reason's stats."""
    return ctx.step_u(opts)


def VF_StepV(ctx, opts=None):
    """VF_StepV (VFMech.c:3057): returns 0 or the negative SNES reason, as the reference."""
    rc, st = ctx.step_v(opts)
    return st["reason"] if st["reason"] < 0 else 0


def VF_UEnergy3D(ctx):
    """(ElasticEnergy, InsituWork, PressureWork) (VFMech.c:1111)."""
    return ctx.u_energy()


def VF_VEnergy3D(ctx):
    """SurfaceEnergy (VFMech.c:2474)."""
    return ctx.v_energy()


def VolumetricCrackOpening(ctx):
    """Crack opening volume (VFPermfield.c:75)."""
    return ctx.crack_opening()


def VFTimeStepPrepare(ctx):
    """VFCommon.c:1132."""
    ctx.time_step_prepare()
