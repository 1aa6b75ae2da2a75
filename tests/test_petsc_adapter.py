"""Compile-only check of the PETSc-side adapter (vpfhf_b200/petsc/VFMech_gpu.c) against the
reference's own headers and a stub of the PETSc declarations it uses.  PETSc is not
installed here, so nothing is linked or run.  The VPFHF source tree is given by the
VPFHF_REFERENCE environment variable; the test is skipped without it."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("VPFHF_REFERENCE", "")


@pytest.mark.skipif(not (REF and os.path.exists(os.path.join(REF, "VFCommon.h"))),
                    reason="VPFHF_REFERENCE does not name the reference source tree")
def test_adapter_compiles_against_reference_headers():
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else shutil.which("gcc")
    cmd = [cc, "-std=c99", "-Wall", "-Werror", "-Wno-unused-variable", "-Wno-unused-function",
           "-fsyntax-only", "-I", os.path.join(ROOT, "tests", "stubs"), "-I", REF,
           "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "vpfhf_b200", "petsc", "VFMech_gpu.c")]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
