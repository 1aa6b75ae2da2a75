"""Oracle fixture for the 129^3 pressurized penny crack (10 AM iterations, AT1): the
FP64-vs-mixed configuration of the benchmark, checked against the FP64 oracle.

The CPU oracle (oracle/) needs about an hour on 8 host cores for this case, so its
results are stored in penny129.npz and compared against by tests/test_gpu_solve.py.
Regenerate from the repository root with

    python tests/golden/make_penny129.py [threads]

Problem: cube [0,4]^3, 129^3 nodes (h = 1/32), E = 1e10, nu = 0.25, Gc = 100, AT1,
epsilon = 2h, eta = 1e-8, one penny crack at (2,2,2), r = 0.4, normal z, thickness 0
(VFCracks.c:185-227); p = 1e6 with crack pressure; rollers on all faces
(BCfiles/3DRollers.txt); CG + Jacobi, rtol 1e-8 (ValidationTests/test18.c:188-220
with the configuration's options).  Per AM iteration the record holds the elastic
energy, pressure work, surface energy, crack opening, ||V - Vold||_inf, the U and V
Krylov and Newton iteration counts and the seconds the oracle spent on the
iteration (its StepU + StepV on the host cores: the CPU AM-step time).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_penny41 import run  # noqa: E402

PARAMS = dict(n=(129, 129, 129), l=(4.0, 4.0, 4.0), E=1e10, nu=0.25, Gc=100.0, atnum=1,
              epsilon=2 * 4.0 / 128, eta=1e-8, center=(2.0, 2.0, 2.0), r=0.4, p=1e6, am_its=10)


if __name__ == "__main__":
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else 0
    t0 = time.time()
    rec, U, V = run(dict(PARAMS, nthreads=threads), log=lambda s: print(s, flush=True))
    np.savez_compressed(os.path.join(HERE, "penny129.npz"), rec=rec, V=V,
                        threads=threads or os.cpu_count(),
                        columns=np.array(["elastic", "pressure_work", "surface", "cov", "errV",
                                          "kspU", "newtonU", "kspV", "newtonV", "seconds"]))
    print(f"done in {time.time() - t0:.0f} s")
