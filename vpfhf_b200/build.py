"""Builds vpfhf_b200/libvfgpu.so (the C-ABI library) with nvcc for sm_100a.

    python -m vpfhf_b200.build [--force] [--debug]

Objects go to vpfhf_b200/_build/; the shared library is written in-tree next to
this file so that it travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvfgpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
# Per-file extra flags: the crack initialisers and the fracture width round like the
# reference's C code.
FILE_FLAGS = {"cracks.cu": ["-fmad=false"], "width.cu": ["-fmad=false"]}


def _flags(debug: bool) -> list[str]:
    f = ARCH + ["-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX,
                "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
    f += ["-O0", "-G"] if debug else ["-O3"]
    return f


def _deps_mtime() -> float:
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hdrs.append(os.path.join(HERE, "..", "include", "vfgpu.h"))
    return max(os.path.getmtime(h) for h in hdrs if os.path.exists(h))


def _compile(src: str, obj: str, debug: bool) -> tuple[str, int, str]:
    cmd = [NVCC] + _flags(debug) + FILE_FLAGS.get(os.path.basename(src), []) + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    return src, p.returncode, p.stdout + p.stderr


def build(force: bool = False, debug: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_t = _deps_mtime()
    jobs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t):
            jobs.append((s, o))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for src, rc, out in ex.map(lambda j: _compile(j[0], j[1], debug), jobs):
                if verbose or rc:
                    sys.stderr.write(f"[nvcc] {os.path.basename(src)}\n{out}")
                if rc:
                    raise RuntimeError(f"nvcc failed on {src}")
    objs = [os.path.join(BUILD, os.path.basename(s)[:-3] + ".o") for s in srcs]
    if jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(map(os.path.getmtime, objs)):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-o", LIB] + objs + ["-cudart", "static"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode:
            raise RuntimeError("link failed:\n" + p.stdout + p.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, debug=a.debug, verbose=a.verbose))
