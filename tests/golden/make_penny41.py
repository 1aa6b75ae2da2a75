"""Oracle fixture for the 41^3 pressurized penny crack (5 AM iterations, AT1).

The CPU oracle (oracle/) is too slow to rerun inside every GPU test session, so its
results for this case are stored in penny41.npz and compared against by
tests/test_gpu_solve.py.  Regenerate from the repository root with

    python tests/golden/make_penny41.py

Problem (ValidationTests/test18.c semantics with the penny-crack options of the
41^3 case): cube [0,4]^3, 41^3 nodes, E = 1e10, nu = 0.25, Gc = 100, AT1,
epsilon = 0.2 (2h), eta = 1e-8, one penny crack at (2,2,2), r = 0.4, normal z,
thickness 0; p = 1e6 with crack pressure; rollers on all faces (3DRollers.txt);
CG + Jacobi, rtol 1e-8.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import vforacle as vo  # noqa: E402

PARAMS = dict(n=(41, 41, 41), l=(4.0, 4.0, 4.0), E=1e10, nu=0.25, Gc=100.0, atnum=1,
              epsilon=0.2, eta=1e-8, center=(2.0, 2.0, 2.0), r=0.4, p=1e6, am_its=5)


def run(P=PARAMS, log=print):
    o = vo.Oracle(P["n"], P["l"], E=P["E"], nu=P["nu"], Gc=P["Gc"], epsilon=P["epsilon"],
                  eta=P["eta"], atnum=P["atnum"], pressurize=True, nthreads=P.get("nthreads", 0))
    N = o.N
    V = o.penny_v(P["center"], P["r"])
    virrev = V.copy()
    U = np.zeros(3 * N)
    p = np.full(N, P["p"])
    umask, uval = o.bc(vo.rollers_face())
    U[umask == 1] = uval[umask == 1]
    lb, ub = np.zeros(N), virrev.copy()
    rec = []
    for it in range(P["am_its"]):
        t0 = time.time()
        vold = V.copy()
        su = o.step_u(U, V, p=p, mask=umask, value=uval)
        sv = o.step_v(V, U, lb, ub, p=p)
        el, pw = o.u_energy(U, V, p=p)
        rec.append([el, pw, o.v_energy(V), o.cov(U, V), np.abs(V - vold).max(),
                    su.ksp_its, su.newton_its, sv.ksp_its, sv.newton_its, time.time() - t0])
        log(f"AM {it}: elastic {el:.9e} pw {pw:.9e} surf {rec[-1][2]:.9e} cov {rec[-1][3]:.9e} "
            f"errV {rec[-1][4]:.3e} kspU {su.ksp_its} kspV {sv.ksp_its} ({time.time() - t0:.1f}s)")
    return np.array(rec), U, V


if __name__ == "__main__":
    rec, U, V = run()
    np.savez_compressed(os.path.join(HERE, "penny41.npz"), rec=rec, V=V, U=U,
                        columns=np.array(["elastic", "pressure_work", "surface", "cov", "errV",
                                          "kspU", "newtonU", "kspV", "newtonV", "seconds"]))
