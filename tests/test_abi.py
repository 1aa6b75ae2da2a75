"""The C-ABI library loads and exports every function include/vfgpu.h declares
(no CUDA calls: runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "vfgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vfgpu_\w+)\s*\(", src)))


def test_library_exports_header():
    from vpfhf_b200 import _abi
    lib = ctypes.CDLL(_abi.LIBPATH)
    names = declared()
    assert "vfgpu_u_apply" in names and "vfgpu_create" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares exactly the header's functions
    assert sorted(_abi.exported_symbols()) == names
