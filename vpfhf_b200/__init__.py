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

__all__ = ["VFContext", "BCSpec", "rollers", "FP64", "MIXED", "VFGPUError"]


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
