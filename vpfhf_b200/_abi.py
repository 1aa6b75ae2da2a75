"""ctypes binding of libvfgpu.so (include/vfgpu.h).

The library is required: on a machine with a CUDA GPU, loading fails loudly if
libvfgpu.so is missing or does not load; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libvfgpu.so")

OK, NOT_CONVERGED, DIVERGED = 0, 1, 2
ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_STATE = -1, -2, -3, -4
FP64, MIXED = 0, 1
UNILATERAL_NONE, UNILATERAL_NOCOMPRESSION = 0, 1
PC_JACOBI, PC_MG, PC_AUTO = 0, 1, 2
BC_NONE, BC_ZERO, BC_ONE, BC_FIXED = 0, 1, 2, 3
FIELD_U, FIELD_V, FIELD_VIRREV, FIELD_BCU, FIELD_THETA, FIELD_THETAREF, FIELD_PRESSURE = range(7)
FIELD_NAMES = {"U": FIELD_U, "V": FIELD_V, "VIrrev": FIELD_VIRREV, "BCU": FIELD_BCU,
               "theta": FIELD_THETA, "thetaRef": FIELD_THETAREF, "pressure": FIELD_PRESSURE}


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double)]


class MatProp(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("alpha", C.c_double),
                ("beta", C.c_double), ("Gc", C.c_double)]


class VFProp(C.Structure):
    _fields_ = [("epsilon", C.c_double), ("eta", C.c_double), ("irrevtol", C.c_double),
                ("atnum", C.c_int), ("hasCrackPressure", C.c_int)]


class BC(C.Structure):
    _fields_ = [("face", C.c_int * 6), ("faceValue", C.c_double * 6),
                ("vertex", C.c_int * 8), ("vertexValue", C.c_double * 8)]


class SolveOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("ksp_rtol", C.c_double), ("ksp_atol", C.c_double),
                ("ksp_dtol", C.c_double), ("ksp_maxit", C.c_int), ("snes_rtol", C.c_double),
                ("snes_atol", C.c_double), ("snes_stol", C.c_double), ("snes_maxit", C.c_int),
                ("inner_rtol", C.c_double), ("max_refine", C.c_int), ("time_limit", C.c_double),
                ("pc", C.c_int)]


class WidthOpts(C.Structure):
    _fields_ = [("int_length", C.c_double), ("width_tol", C.c_double),
                ("remove_tip_effect", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("newton_its", C.c_int), ("ksp_its", C.c_int), ("refine_its", C.c_int),
                ("reason", C.c_int), ("fnorm0", C.c_double), ("fnorm", C.c_double),
                ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Penny(C.Structure):
    _fields_ = [("center", C.c_double * 3), ("r", C.c_double), ("theta", C.c_double),
                ("phi", C.c_double), ("thickness", C.c_double)]


class Rect(C.Structure):
    _fields_ = [("corners", C.c_double * 9), ("thickness", C.c_double)]


SERVE_MAX_PENNY = 16
SERVE_MAX_RECT = 16


class Request(C.Structure):
    _fields_ = [("grid", Grid), ("mp", MatProp), ("vf", VFProp), ("bcU", BC * 3), ("bcV", BC),
                ("pressure", C.c_double), ("npenny", C.c_int), ("nrect", C.c_int),
                ("penny", Penny * SERVE_MAX_PENNY), ("rect", Rect * SERVE_MAX_RECT),
                ("am_its", C.c_int), ("altmintol", C.c_double), ("max_am_its", C.c_int),
                ("opts", SolveOpts), ("out_u", C.c_void_p), ("out_v", C.c_void_p),
                ("out_cellcov", C.c_void_p), ("tag", C.c_ulonglong)]


class Result(C.Structure):
    _fields_ = [("ticket", C.c_ulonglong), ("tag", C.c_ulonglong), ("status", C.c_int),
                ("am_its", C.c_int), ("ksp_its_u", C.c_int), ("ksp_its_v", C.c_int),
                ("am_err", C.c_double), ("elastic", C.c_double), ("pressure_work", C.c_double),
                ("surface", C.c_double), ("cov", C.c_double), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_done", C.c_double), ("worker", C.c_int),
                ("reused_ctx", C.c_int), ("error", C.c_char * 160)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["error"] = self.error.decode(errors="replace")
        return d


class ServerInfo(C.Structure):
    _fields_ = [("budget_bytes", C.c_longlong), ("reserved_bytes", C.c_longlong),
                ("peak_reserved_bytes", C.c_longlong), ("workers", C.c_int),
                ("contexts", C.c_int), ("contexts_created", C.c_int), ("evictions", C.c_int),
                ("submitted", C.c_longlong), ("completed", C.c_longlong),
                ("queued", C.c_longlong), ("running", C.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class VFGPUError(RuntimeError):
    def __init__(self, code, fn, msg):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


_LIB = None

# name -> argtypes (all return int)
_SIGS = {
    "vfgpu_create": [C.POINTER(Grid), C.POINTER(C.c_void_p)],
    "vfgpu_destroy": [C.c_void_p],
    "vfgpu_memory_estimate": [C.POINTER(Grid), C.POINTER(C.c_longlong)],
    "vfgpu_mg_hierarchy": [C.POINTER(Grid), C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                           C.POINTER(C.c_longlong)],
    "vfgpu_set_matprop": [C.c_void_p, C.c_int, C.POINTER(MatProp), C.c_void_p],
    "vfgpu_set_cell_modulus": [C.c_void_p, C.c_void_p],
    "vfgpu_set_vfprop": [C.c_void_p, C.POINTER(VFProp)],
    "vfgpu_set_bc": [C.c_void_p, C.POINTER(BC), C.POINTER(BC)],
    "vfgpu_set_insitu": [C.c_void_p, C.c_void_p, C.c_void_p],
    "vfgpu_set_unilateral": [C.c_void_p, C.c_int],
    "vfgpu_set_u_split": [C.c_void_p, C.c_int],
    "vfgpu_set_field": [C.c_void_p, C.c_int, C.c_void_p],
    "vfgpu_get_field": [C.c_void_p, C.c_int, C.c_void_p],
    "vfgpu_u_apply": [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p],
    "vfgpu_u_apply_dev": [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p],
    "vfgpu_get_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
    "vfgpu_step_u": [C.c_void_p, C.POINTER(SolveOpts), C.POINTER(SolveStats)],
    "vfgpu_step_v": [C.c_void_p, C.POINTER(SolveOpts), C.POINTER(SolveStats)],
    "vfgpu_time_step_prepare": [C.c_void_p],
    "vfgpu_am_step": [C.c_void_p, C.POINTER(SolveOpts), C.POINTER(C.c_double),
                      C.POINTER(SolveStats), C.POINTER(SolveStats)],
    "vfgpu_u_energy": [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                       C.POINTER(C.c_double)],
    "vfgpu_v_energy": [C.c_void_p, C.POINTER(C.c_double)],
    "vfgpu_crack_opening": [C.c_void_p, C.POINTER(C.c_double), C.c_void_p],
    "vfgpu_u_residual": [C.c_void_p, C.c_void_p],
    "vfgpu_v_residual": [C.c_void_p, C.c_void_p],
    "vfgpu_init_cracks": [C.c_void_p, C.c_int, C.POINTER(Penny), C.c_int, C.POINTER(Rect)],
    "vfgpu_update_fracture_width": [C.c_void_p, C.POINTER(WidthOpts), C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.POINTER(C.c_int)],
    "vfgpu_fracture_well_rate": [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)],
    "vfgpu_cell_to_node": [C.c_void_p, C.c_void_p, C.c_void_p],
    "vfgpu_server_create": [C.c_int, C.c_int, C.c_longlong, C.POINTER(C.c_void_p)],
    "vfgpu_server_submit": [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_ulonglong)],
    "vfgpu_server_next": [C.c_void_p, C.c_double, C.POINTER(Result)],
    "vfgpu_server_info_get": [C.c_void_p, C.POINTER(ServerInfo)],
    "vfgpu_server_destroy": [C.c_void_p],
    "vfgpu_fma_peak": [C.c_int, C.POINTER(C.c_double)],
    "vfgpu_u_apply_tc": [C.c_void_p, C.c_void_p, C.c_void_p],
    "vfgpu_tc_error": [C.c_void_p, C.POINTER(C.c_int)],
    "vfgpu_tc_tables": [C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p],
    "vfgpu_wait_selftest": [C.c_longlong, C.c_int, C.POINTER(C.c_int)],
    "vfgpu_u_apply_noalloc": [C.POINTER(Grid), C.POINTER(MatProp), C.c_double, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
}
_VOID_SIGS = {"vfgpu_default_solve_opts": [C.POINTER(SolveOpts)],
              "vfgpu_default_width_opts": [C.POINTER(WidthOpts)]}


def lib():
    """Loads libvfgpu.so (building it first if the sources are present and it is missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIBPATH):
        from . import build as _build
        _build.build()
    L = C.CDLL(LIBPATH)
    L.vfgpu_last_error.restype = C.c_char_p
    L.vfgpu_last_error.argtypes = []
    for name, args in _SIGS.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    for name, args in _VOID_SIGS.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = None
    L.vfgpu_server_clock.argtypes = [C.c_void_p]
    L.vfgpu_server_clock.restype = C.c_double
    _LIB = L
    return L


def exported_symbols():
    return ["vfgpu_last_error", "vfgpu_server_clock"] + list(_SIGS) + list(_VOID_SIGS)


def check(code, fn):
    if code < 0:
        raise VFGPUError(code, fn, lib().vfgpu_last_error().decode())
    return code


def ptr(a):
    """Raw address of a numpy array (host) or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return a.data_ptr()  # torch.Tensor
