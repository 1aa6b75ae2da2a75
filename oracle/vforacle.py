"""ctypes binding of the CPU oracle (oracle/libvforacle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker and by bench.py's CPU-baseline leg.  The product path (vpfhf_b200)
never imports this module.

The oracle restates the reference's FP64 arithmetic (VFCartFE.c, VFMech.c,
VFCracks.c, VFPermfield.c, VFCommon.c); see oracle/vf_oracle.h for the
per-function citations.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

NONE, ZERO, ONE, FIXED = 0, 1, 2, 3
MAXLAYER = 16


def build():
    """Compile oracle/libvforacle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libvforacle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _declare(_LIB)
    return _LIB


class Problem(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("nlayer", C.c_int),
        ("E", C.c_double * MAXLAYER), ("nu", C.c_double * MAXLAYER),
        ("alpha", C.c_double * MAXLAYER), ("beta", C.c_double * MAXLAYER),
        ("Gc", C.c_double * MAXLAYER),
        ("layer", C.POINTER(C.c_int)),
        ("cellE", C.POINTER(C.c_double)),
        ("epsilon", C.c_double), ("eta", C.c_double), ("irrevtol", C.c_double),
        ("atnum", C.c_int), ("hasCrackPressure", C.c_int), ("nthreads", C.c_int),
        ("hasInsitu", C.c_int), ("insitumin", C.c_double * 6), ("insitumax", C.c_double * 6),
        ("insitu_free", (C.c_int * 3) * 6), ("unilateral", C.c_int),
    ]


class SolverOpts(C.Structure):
    _fields_ = [
        ("rtol", C.c_double), ("atol", C.c_double), ("dtol", C.c_double), ("maxit", C.c_int),
        ("snes_rtol", C.c_double), ("snes_atol", C.c_double), ("snes_stol", C.c_double),
        ("snes_maxit", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [("newton_its", C.c_int), ("ksp_its", C.c_int), ("reason", C.c_int),
                ("fnorm0", C.c_double), ("fnorm", C.c_double)]


def default_opts(maxit=100000):
    """KSP/SNES tolerances the reference sets (VFCommon.c:1024,1039,1071,1081)."""
    return SolverOpts(1e-8, 1e-10, 1e5, maxit, 1e-8, 1e-8, 1e-8, 50)


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_P = C.POINTER(Problem)


class _Opt:
    """Accepts a numpy array or None for optional pointer arguments."""

    def __init__(self, dt):
        self.dt = dt

    def from_param(self, obj):
        if obj is None:
            return None
        return np.ctypeslib.as_ctypes(np.ascontiguousarray(obj, dtype=self.dt))


def _declare(L):
    odp, ou8 = _Opt(np.float64), _Opt(np.uint8)
    sig = {
        "vfo_tables": [C.c_double, C.c_double, C.c_double, _dp, _dp, _dp],
        "vfo_bc_build": [C.c_int, C.c_int, C.c_int, C.c_int, _i32, _i32, odp, _u8, _dp],
        "vfo_u_element_matrix": [_P, C.c_int, C.c_int, C.c_int, _dp, _dp],
        "vfo_u_apply_ref": [_P, _dp, _dp, ou8, _dp],
        "vfo_u_apply_mf": [_P, _dp, _dp, ou8, _dp],
        "vfo_u_rhs": [_P, _dp, odp, odp, odp, _dp],
        "vfo_u_residual_ref": [_P, _dp, _dp, odp, odp, odp, ou8, odp, _dp],
        "vfo_u_diag": [_P, _dp, ou8, _dp],
        "vfo_u_assemble_csr": [_P, _dp, ou8, _i64, _i32, _dp],
        "vfo_csr_spmv": [C.c_int64, _i64, _i32, _dp, _dp, _dp, C.c_int],
        "vfo_v_element_matrix": [_P, C.c_int, C.c_int, C.c_int, _dp, odp, odp, _dp],
        "vfo_v_rhs": [_P, _dp, odp, _dp],
        "vfo_v_residual_ref": [_P, _dp, _dp, odp, odp, odp, odp, ou8, odp, _dp],
        "vfo_v_apply": [_P, _dp, odp, odp, odp, ou8, _dp, _dp],
        "vfo_v_diag": [_P, _dp, odp, odp, odp, ou8, _dp],
        "vfo_u_energy": [_P, _dp, _dp, odp, odp, odp, _dp],
        "vfo_v_energy": [_P, _dp, C.POINTER(C.c_double)],
        "vfo_cov": [_P, _dp, _dp, C.POINTER(C.c_double), odp],
        "vfo_penny_crack_v": [_P, _dp, C.c_double, C.c_double, C.c_double, C.c_double, _dp],
        "vfo_rect_crack_v": [_P, _dp, C.c_double, _dp],
        "vfo_cracks_v": [_P, C.c_int, odp, C.c_int, odp, _dp],
        "vfo_insitu_work": [_P, _dp, C.POINTER(C.c_double)],
        "vfo_u_apply_mf_u": [_P, odp, _dp, _dp, ou8, _dp],
        "vfo_u_apply_ref_u": [_P, odp, _dp, _dp, ou8, _dp],
        "vfo_u_rhs_u": [_P, odp, _dp, odp, odp, odp, _dp],
        "vfo_u_diag_u": [_P, odp, _dp, ou8, _dp],
        "vfo_fracture_width": [_P, _dp, _dp, C.c_double, C.c_double, C.c_int, _dp, _dp,
                               C.POINTER(C.c_int)],
        "vfo_cell_to_node": [_P, _dp, _dp],
        "vfo_fracture_well_rate": [_P, _dp, _dp, C.POINTER(C.c_double)],
        "vfo_step_u": [_P, _dp, _dp, odp, odp, odp, ou8, odp, C.POINTER(SolverOpts),
                       C.POINTER(Stats)],
        "vfo_step_v": [_P, _dp, _dp, odp, odp, odp, odp, _dp, _dp, ou8, odp,
                       C.POINTER(SolverOpts), C.POINTER(Stats)],
        "vfo_step_u_asm": [_P, _dp, _dp, odp, odp, odp, ou8, odp, C.POINTER(SolverOpts),
                           C.POINTER(Stats), C.POINTER(C.c_double)],
        "vfo_step_v_asm": [_P, _dp, _dp, odp, odp, odp, odp, _dp, _dp, ou8, odp,
                           C.POINTER(SolverOpts), C.POINTER(Stats), C.POINTER(C.c_double)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.vfo_rect_distance.argtypes = [_dp, _dp]
    L.vfo_rect_distance.restype = C.c_double
    L.vfo_width_int_length.argtypes = [_P]
    L.vfo_width_int_length.restype = C.c_double
    L.vfo_u_csr_nnz.argtypes = [_P]
    L.vfo_u_csr_nnz.restype = C.c_int64


class Oracle:
    """One problem instance: grid, per-layer material, phase-field parameters."""

    def __init__(self, n, l, E=1.0, nu=0.0, Gc=1.0, alpha=0.0, beta=0.0, epsilon=0.2,
                 eta=1e-8, atnum=1, irrevtol=5e-2, pressurize=True, cellE=None, layer=None,
                 nthreads=0, unilateral=0):
        L = lib()
        self.L = L
        nx, ny, nz = (int(x) for x in n)
        self.n = (nx, ny, nz)
        self.N = nx * ny * nz
        P = Problem()
        P.nx, P.ny, P.nz = nx, ny, nz
        P.lx, P.ly, P.lz = (float(x) for x in l)
        Es, nus = np.atleast_1d(E), np.atleast_1d(nu)
        P.nlayer = len(Es)
        for k in range(P.nlayer):
            P.E[k] = float(Es[k])
            P.nu[k] = float(np.broadcast_to(nus, Es.shape)[k])
            P.alpha[k] = float(np.broadcast_to(np.atleast_1d(alpha), Es.shape)[k])
            P.beta[k] = float(np.broadcast_to(np.atleast_1d(beta), Es.shape)[k])
            P.Gc[k] = float(np.broadcast_to(np.atleast_1d(Gc), Es.shape)[k])
        self._layer = None if layer is None else np.ascontiguousarray(layer, dtype=np.int32)
        self._cellE = None if cellE is None else np.ascontiguousarray(cellE, dtype=np.float64)
        P.layer = (self._layer.ctypes.data_as(C.POINTER(C.c_int)) if self._layer is not None
                   else None)
        P.cellE = (self._cellE.ctypes.data_as(C.POINTER(C.c_double)) if self._cellE is not None
                   else None)
        P.epsilon, P.eta, P.irrevtol = float(epsilon), float(eta), float(irrevtol)
        P.atnum, P.hasCrackPressure, P.nthreads = int(atnum), int(bool(pressurize)), int(nthreads)
        P.unilateral = int(unilateral)
        self.P = P

    # -- helpers ---------------------------------------------------------
    def zeros(self, dof=1):
        return np.zeros(self.N * dof)

    def bc(self, face, vertex=None, dof=3, bcu=None):
        """face/vertex: arrays [dof][6] / [dof][8] of BC types -> (mask, value)."""
        face = np.ascontiguousarray(np.asarray(face, dtype=np.int32).reshape(dof, 6))
        vertex = np.zeros((dof, 8), np.int32) if vertex is None else np.asarray(vertex, np.int32)
        vertex = np.ascontiguousarray(vertex.reshape(dof, 8))
        mask = np.zeros(self.N * dof, np.uint8)
        value = np.zeros(self.N * dof)
        self.L.vfo_bc_build(*self.n, dof, face, vertex, bcu, mask, value)
        return mask, value

    # -- U ---------------------------------------------------------------
    def u_apply_ref(self, v, x, mask=None):
        y = np.zeros(3 * self.N)
        self.L.vfo_u_apply_ref(C.byref(self.P), v, x, mask, y)
        return y

    def u_apply(self, v, x, mask=None):
        y = np.zeros(3 * self.N)
        self.L.vfo_u_apply_mf(C.byref(self.P), v, x, mask, y)
        return y

    def u_rhs(self, v, theta=None, thetaRef=None, p=None):
        f = np.zeros(3 * self.N)
        self.L.vfo_u_rhs(C.byref(self.P), v, theta, thetaRef, p, f)
        return f

    def u_residual_ref(self, u, v, theta=None, thetaRef=None, p=None, mask=None, value=None):
        F = np.zeros(3 * self.N)
        self.L.vfo_u_residual_ref(C.byref(self.P), u, v, theta, thetaRef, p, mask, value, F)
        return F

    def u_diag(self, v, mask=None):
        d = np.zeros(3 * self.N)
        self.L.vfo_u_diag(C.byref(self.P), v, mask, d)
        return d

    def u_element_matrix(self, ei, ej, ek, v):
        K = np.zeros(576)
        self.L.vfo_u_element_matrix(C.byref(self.P), ei, ej, ek, v, K)
        return K.reshape(24, 24)

    def u_csr(self, v, mask=None):
        nnz = self.L.vfo_u_csr_nnz(C.byref(self.P))
        rowptr = np.zeros(3 * self.N + 1, np.int64)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        self.L.vfo_u_assemble_csr(C.byref(self.P), v, mask, rowptr, col, val)
        return rowptr, col, val

    def csr_spmv(self, csr, x, nthreads=0):
        rowptr, col, val = csr
        y = np.zeros(len(rowptr) - 1)
        self.L.vfo_csr_spmv(len(rowptr) - 1, rowptr, col, val, x, y, nthreads)
        return y

    # -- V ---------------------------------------------------------------
    def v_rhs(self, u, p=None):
        b = np.zeros(self.N)
        self.L.vfo_v_rhs(C.byref(self.P), u, p, b)
        return b

    def v_residual_ref(self, u, v, theta=None, thetaRef=None, p=None, virrev=None, mask=None,
                       value=None):
        F = np.zeros(self.N)
        self.L.vfo_v_residual_ref(C.byref(self.P), u, v, theta, thetaRef, p, virrev, mask, value,
                                  F)
        return F

    def v_apply(self, u, x, theta=None, thetaRef=None, virrev=None, mask=None):
        y = np.zeros(self.N)
        self.L.vfo_v_apply(C.byref(self.P), u, theta, thetaRef, virrev, mask, x, y)
        return y

    def v_diag(self, u, theta=None, thetaRef=None, virrev=None, mask=None):
        d = np.zeros(self.N)
        self.L.vfo_v_diag(C.byref(self.P), u, theta, thetaRef, virrev, mask, d)
        return d

    def v_element_matrix(self, ei, ej, ek, u, theta=None, thetaRef=None):
        K = np.zeros(64)
        self.L.vfo_v_element_matrix(C.byref(self.P), ei, ej, ek, u, theta, thetaRef, K)
        return K.reshape(8, 8)

    # -- energies ----------------------------------------------------------
    def u_energy(self, u, v, theta=None, thetaRef=None, p=None):
        out = np.zeros(2)
        self.L.vfo_u_energy(C.byref(self.P), u, v, theta, thetaRef, p, out)
        return float(out[0]), float(out[1])

    def v_energy(self, v):
        s = C.c_double()
        self.L.vfo_v_energy(C.byref(self.P), v, C.byref(s))
        return s.value

    def cov(self, u, v, cell=False):
        c = C.c_double()
        cc = np.zeros((self.n[0] - 1) * (self.n[1] - 1) * (self.n[2] - 1)) if cell else None
        self.L.vfo_cov(C.byref(self.P), u, v, C.byref(c), cc)
        return (c.value, cc) if cell else c.value

    def width_int_length(self):
        """VFCtx.WidthIntLenght = 3 res + 4 epsilon (VFCommon.c:897-914)."""
        return self.L.vfo_width_int_length(C.byref(self.P))

    def fracture_width(self, u, v, int_length=None, width_tol=0.1, remove_tip=False):
        """UpdateFractureWidth (VFPermfield.c:267-562) + CellToNodeInterpolation:
        returns (widthc per cell, width per node, pmult per cell, stalled band cells)."""
        nc = (self.n[0] - 1) * (self.n[1] - 1) * (self.n[2] - 1)
        wc, pm, st = np.zeros(nc), np.zeros(nc), C.c_int()
        L = self.width_int_length() if int_length is None else float(int_length)
        self.L.vfo_fracture_width(C.byref(self.P), np.ascontiguousarray(u, np.float64),
                                  np.ascontiguousarray(v, np.float64), L, float(width_tol),
                                  int(bool(remove_tip)), wc, pm, C.byref(st))
        return wc, self.cell_to_node(wc), pm, st.value

    def cell_to_node(self, cellv):
        out = np.zeros(self.N)
        self.L.vfo_cell_to_node(C.byref(self.P), np.ascontiguousarray(cellv, np.float64), out)
        return out

    def fracture_well_rate(self, v, regrate):
        """VolumetricFractureWellRate (VFPermfield.c:1513-1604)."""
        r = C.c_double()
        self.L.vfo_fracture_well_rate(C.byref(self.P), np.ascontiguousarray(v, np.float64),
                                      np.ascontiguousarray(regrate, np.float64), C.byref(r))
        return r.value

    def penny_v(self, center, r, theta=0.0, phi=0.0, thickness=0.0):
        v = np.zeros(self.N)
        self.L.vfo_penny_crack_v(C.byref(self.P), np.asarray(center, np.float64), float(r),
                                 float(theta), float(phi), float(thickness), v)
        return v

    def set_insitu(self, smin, smax=None, face_bc=None):
        """In-situ stresses (Voigt s11 s22 s33 s23 s13 s12) at z = 0 and z = lz; face_bc:
        [3][6] U BC types per component and face (X0 X1 Y0 Y1 Z0 Z1), traction only
        where the type is NONE.  smin=None switches them off."""
        P = self.P
        P.hasInsitu = int(smin is not None)
        if smin is None:
            return
        smax = smin if smax is None else smax
        for i in range(6):
            P.insitumin[i], P.insitumax[i] = float(smin[i]), float(smax[i])
        fb = np.zeros((3, 6), int) if face_bc is None else np.asarray(face_bc).reshape(3, 6)
        for f in range(6):
            for c in range(3):
                P.insitu_free[f][c] = int(fb[c, f] == NONE)

    def insitu_work(self, u):
        w = C.c_double()
        self.L.vfo_insitu_work(C.byref(self.P), u, C.byref(w))
        return w.value

    def u_apply_u(self, u0, v, x, mask=None, ref=False):
        """K(v; u0) x: the operator linearised at u0 (NOCOMPRESSION sign pattern)."""
        y = np.zeros(3 * self.N)
        f = self.L.vfo_u_apply_ref_u if ref else self.L.vfo_u_apply_mf_u
        f(C.byref(self.P), u0, v, x, mask, y)
        return y

    def u_rhs_u(self, u0, v, theta=None, thetaRef=None, p=None):
        f = np.zeros(3 * self.N)
        self.L.vfo_u_rhs_u(C.byref(self.P), u0, v, theta, thetaRef, p, f)
        return f

    def u_diag_u(self, u0, v, mask=None):
        d = np.zeros(3 * self.N)
        self.L.vfo_u_diag_u(C.byref(self.P), u0, v, mask, d)
        return d

    def rect_v(self, corners, thickness=0.0):
        v = np.zeros(self.N)
        self.L.vfo_rect_crack_v(C.byref(self.P), np.asarray(corners, np.float64), float(thickness), v)
        return v

    def rect_distance(self, x, corners):
        return self.L.vfo_rect_distance(np.asarray(x, np.float64), np.asarray(corners, np.float64))

    def cracks_v(self, pennies=(), rects=()):
        """pennies: rows (cx, cy, cz, r, theta, phi, thickness); rects: rows (9 corners,
        thickness).  V = VIrrev = the pointwise minimum (VFCommon.c:823-857)."""
        pa = np.ascontiguousarray(np.asarray(pennies, np.float64).reshape(-1, 7))
        ra = np.ascontiguousarray(np.asarray(rects, np.float64).reshape(-1, 10))
        v = np.zeros(self.N)
        self.L.vfo_cracks_v(C.byref(self.P), len(pa), pa if len(pa) else None, len(ra),
                            ra if len(ra) else None, v)
        return v

    # -- solvers -------------------------------------------------------------
    def step_u(self, u, v, theta=None, thetaRef=None, p=None, mask=None, value=None, opts=None):
        st = Stats()
        o = opts or default_opts()
        self.L.vfo_step_u(C.byref(self.P), u, v, theta, thetaRef, p, mask, value, C.byref(o),
                          C.byref(st))
        return st

    def step_v(self, v, u, lb, ub, theta=None, thetaRef=None, p=None, virrev=None, mask=None,
               value=None, opts=None):
        st = Stats()
        o = opts or default_opts()
        self.L.vfo_step_v(C.byref(self.P), v, u, theta, thetaRef, p, virrev,
                          np.ascontiguousarray(lb, np.float64), np.ascontiguousarray(ub, np.float64),
                          mask, value, C.byref(o), C.byref(st))
        return st


    def step_u_asm(self, u, v, theta=None, thetaRef=None, p=None, mask=None, value=None,
                   opts=None):
        """StepU by the reference's method (assembled Jacobian, CG on the CSR matrix);
        returns (stats, seconds spent assembling)."""
        st, ta = Stats(), C.c_double()
        o = opts or default_opts()
        self.L.vfo_step_u_asm(C.byref(self.P), u, v, theta, thetaRef, p, mask, value, C.byref(o),
                              C.byref(st), C.byref(ta))
        return st, ta.value

    def step_v_asm(self, v, u, lb, ub, theta=None, thetaRef=None, p=None, virrev=None,
                   mask=None, value=None, opts=None):
        st, ta = Stats(), C.c_double()
        o = opts or default_opts()
        self.L.vfo_step_v_asm(C.byref(self.P), v, u, theta, thetaRef, p, virrev,
                              np.ascontiguousarray(lb, np.float64),
                              np.ascontiguousarray(ub, np.float64), mask, value, C.byref(o),
                              C.byref(st), C.byref(ta))
        return st, ta.value


def rollers_face():
    """BCfiles/3DRollers.txt: normal component ZERO on each face."""
    f = np.zeros((3, 6), np.int32)
    f[0, 0] = f[0, 1] = ZERO
    f[1, 2] = f[1, 3] = ZERO
    f[2, 4] = f[2, 5] = ZERO
    return f
