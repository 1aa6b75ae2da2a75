"""Reference driver programs restated for the tests (test infrastructure)."""
from __future__ import annotations

import numpy as np


def runtest1_oracle(vo, steps=11, altmintol=1e-3):
    """ValidationTests/test1.c with the `make runtest1` arguments (makefile:196-198),
    on the CPU oracle.  Returns one record per time step."""
    o = vo.Oracle((101, 5, 5), (10., 1., 1.), E=1.0, nu=0.0, Gc=0.1, epsilon=0.5, eta=1e-8,
                  atnum=1, pressurize=False)
    N = o.N
    face = np.zeros((3, 6), np.int32)
    face[0, 0] = face[0, 1] = vo.FIXED
    face[1, 0] = face[1, 1] = face[2, 0] = face[2, 1] = vo.ZERO
    fv = np.zeros((1, 6), np.int32)
    fv[0, 0] = fv[0, 1] = vo.ONE
    # VecSetFromBC: FIXED faces take faceValue (-1 at X0, +1 at X1), scaled by t
    bcu1 = np.zeros(3 * N)
    X = np.arange(N) % 101
    bcu1[0::3][X == 0] = -1.0
    bcu1[0::3][X == 100] = 1.0
    vmask, vval = o.bc(fv, dof=1)
    U = np.zeros(3 * N)
    V = np.ones(N)
    out = []
    for ts in range(steps):
        t = 0.4 * ts
        umask, uval = o.bc(face, dof=3, bcu=bcu1 * t)
        virrev = V.copy()                        # VFTimeStepPrepare (VFCommon.c:1141)
        U[umask == 1] = uval[umask == 1]         # VecApplyDirichletBC(U)
        V[vmask == 1] = vval[vmask == 1]         # VecApplyDirichletBC(V)
        lb, ub = np.zeros(N), virrev.copy()      # AT1 bounds [0, VIrrev]
        it = 0
        while True:
            vold = V.copy()
            o.step_u(U, V, mask=umask, value=uval)
            o.step_v(V, U, lb, ub, mask=vmask, value=vval)
            err = np.abs(V - vold).max()
            it += 1
            if not (err >= altmintol and it <= 10000):
                break
        cov = o.cov(U, V)
        el, _ = o.u_energy(U, V)
        out.append(dict(t=t, am_its=it, cov=cov, elastic=el, surface=o.v_energy(V)))
    return out
