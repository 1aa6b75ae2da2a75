"""Synthetic inputs of the large configurations: heterogeneous Young's modulus,
pore-pressure fields and random penny cracks, all from seeded generators.

    heterogeneous_modulus   per-cell E = exp(mu_L + 0.5 g), g seeded white noise
                            smoothed by a 3-D Gaussian and renormalised
    pore_pressure           linear gradient in x plus a smooth seeded perturbation
    random_pennies          normals uniform on the sphere, radii and centres uniform
    c3_problem / c5_problem the two large-grid set-ups built from these
"""
from __future__ import annotations

import math

import numpy as np


def _smooth_unit(rng, shape, sigma_cells):
    """White noise N(0,1) on `shape` (z, y, x) smoothed by a Gaussian of standard deviation
    sigma_cells (in cells) and renormalised to zero mean, unit variance."""
    from scipy.ndimage import gaussian_filter
    g = rng.standard_normal(shape).astype(np.float32)
    g = gaussian_filter(g, sigma=sigma_cells, mode="wrap", truncate=3.0)
    g -= g.mean()
    g /= g.std()
    return g


def heterogeneous_modulus(n, seed, mean=1e10, log_sigma=0.5, width_h=8.0):
    """Per-cell E ((nz-1)(ny-1)(nx-1), x fastest): exp(mu_L + log_sigma g) with
    mu_L = ln(mean) - log_sigma^2 / 2, so that the mean of E is `mean`."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    g = _smooth_unit(rng, (nz - 1, ny - 1, nx - 1), width_h)
    mu_l = math.log(mean) - 0.5 * log_sigma ** 2
    return np.exp(mu_l + log_sigma * g.astype(np.float64)).reshape(-1)


def pore_pressure(n, l, seed, p0=10e6, dp=2e6, amp=0.1e6, width_h=8.0):
    """Nodal p = p0 + dp x / lx + amp g, g a smooth unit-variance field."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed + 1)
    g = _smooth_unit(rng, (nz, ny, nx), width_h).astype(np.float64)
    x = np.arange(nx) * (l[0] / (nx - 1))
    return (p0 + dp * x[None, None, :] / l[0] + amp * g).reshape(-1)


def random_pennies(rng, l, count, rmin=0.05, rmax=0.2):
    """Penny cracks (dicts for VFContext.init_cracks): normals uniform on the sphere
    (theta uniform in [0, 360), phi = acos(1 - 2u) in degrees), radius U[rmin, rmax] times
    the shortest box side, centre uniform in the inner 60 % of the box."""
    out = []
    for _ in range(count):
        theta = rng.uniform(0.0, 360.0)
        phi = math.degrees(math.acos(1.0 - 2.0 * rng.uniform()))
        r = rng.uniform(rmin, rmax) * min(l)
        center = [rng.uniform(0.2 * x, 0.8 * x) for x in l]
        out.append(dict(center=center, r=r, theta=theta, phi=phi, thickness=0.0))
    return out


def c3_problem(seed=1003, n=(257, 257, 129), l=(4.0, 4.0, 2.0)):
    """Heterogeneous poroelastic set-up: lognormal E (mean 10 GPa, log-sigma 0.5, 8h
    smoothing), nu 0.25, Biot 0.7, pore pressure 10 -> 12 MPa in x plus a 0.1 MPa smooth
    perturbation acting through the Biot term (no separate crack-pressure term), 16
    random penny cracks, AT1, eps = 2h, eta = 1e-8, Gc = 100."""
    rng = np.random.default_rng(seed)
    h = l[0] / (n[0] - 1)
    return dict(n=n, l=l, cellE=heterogeneous_modulus(n, seed), nu=0.25, beta=0.7, Gc=100.0,
                pressure=pore_pressure(n, l, seed), pennies=random_pennies(rng, l, 16),
                epsilon=2 * h, eta=1e-8, atnum=1, pressurize=False)


def c5_problem(seed=1005, n=(321, 321, 321), l=(4.0, 4.0, 4.0), p=1e6):
    """Large single instance: lognormal E as c3_problem, nu 0.25, 8 random penny cracks
    under a uniform 1 MPa crack pressure, AT1, eps = 2h, eta = 1e-8, Gc = 100."""
    rng = np.random.default_rng(seed)
    h = l[0] / (n[0] - 1)
    return dict(n=n, l=l, cellE=heterogeneous_modulus(n, seed), nu=0.25, beta=0.0, Gc=100.0,
                pressure=np.full(n[0] * n[1] * n[2], p), pennies=random_pennies(rng, l, 8),
                epsilon=2 * h, eta=1e-8, atnum=1, pressurize=True)


def make_context(vg, prob):
    """A VFContext holding `prob` (U = 0, V = VIrrev from the cracks, rollers)."""
    n, l = prob["n"], prob["l"]
    ctx = vg.VFContext(n, l, dict(E=1.0, nu=prob["nu"], beta=prob["beta"], Gc=prob["Gc"]),
                       epsilon=prob["epsilon"], eta=prob["eta"], atnum=prob["atnum"],
                       pressurize=prob["pressurize"])
    ctx.set_cell_modulus(prob["cellE"])
    ctx.set_bc(vg.rollers())
    ctx.set_field("pressure", prob["pressure"])
    ctx.init_cracks(prob["pennies"])
    ctx.time_step_prepare()
    return ctx
