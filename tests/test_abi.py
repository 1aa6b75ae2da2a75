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


def test_struct_layouts_match_header(tmp_path):
    """Every struct the Python binding mirrors has the C compiler's size and field offsets."""
    import shutil
    import subprocess
    from vpfhf_b200 import _abi
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    structs = {"vfgpu_grid": _abi.Grid, "vfgpu_matprop": _abi.MatProp,
               "vfgpu_vfprop": _abi.VFProp, "vfgpu_bc": _abi.BC,
               "vfgpu_solve_opts": _abi.SolveOpts, "vfgpu_solve_stats": _abi.SolveStats,
               "vfgpu_penny": _abi.Penny, "vfgpu_rect": _abi.Rect,
               "vfgpu_request": _abi.Request, "vfgpu_result": _abi.Result,
               "vfgpu_server_info": _abi.ServerInfo, "vfgpu_width_opts": _abi.WidthOpts}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "vfgpu.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
