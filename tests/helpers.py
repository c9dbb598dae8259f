"""Shared helpers of the test suite (comparison norms, halo-filled inputs)."""
from __future__ import annotations

import numpy as np

import oracle
from alpaca_b200 import cases


def filled(case: cases.Case) -> np.ndarray:
    """The case's blocks with face halos and zero-gradient slabs filled by the oracle."""
    u = np.ascontiguousarray(case.u.copy())
    oracle.Restatement(case.grid.dim).halo_update(u, case.grid.nbr)
    return u


def field_rel_err(a: np.ndarray, b: np.ndarray, field_axis: int = 1) -> np.ndarray:
    """Per-field normwise relative error max|a-b| / max|b| (b the reference)."""
    a = np.moveaxis(a, field_axis, 0).reshape(a.shape[field_axis], -1)
    b = np.moveaxis(b, field_axis, 0).reshape(b.shape[field_axis], -1)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return np.abs(a - b).max(axis=1) / scale


def field_rel_err_floored(a: np.ndarray, b: np.ndarray, field_axis: int = 1) -> np.ndarray:
    """field_rel_err, except that a field whose reference is identically zero
    (e.g. the mass right-hand side of a scheme without dissipation on a fluid
    at rest) is measured against the largest field's scale."""
    a2 = np.moveaxis(a, field_axis, 0).reshape(a.shape[field_axis], -1)
    b2 = np.moveaxis(b, field_axis, 0).reshape(b.shape[field_axis], -1)
    scale = np.abs(b2).max(axis=1)
    scale = np.where(scale > 0.0, scale, max(scale.max(), 1e-300))
    return np.abs(a2 - b2).max(axis=1) / scale


def l1_rel(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


def small_cases():
    """Small seeded cases in 1, 2 and 3 dimensions (seconds on the CPU oracle)."""
    return {
        1: cases.sod_1d(),
        2: cases.fourier_shock(2, dim=2, seed=3),
        3: cases.fourier_shock(1, dim=3, seed=5),
    }


# The reference testsuite's DetailedSod error table
# (testsuite/ReferenceValues/DetailedSod/1D_DetailedSod_errors_reference.csv):
# (DensityL1, DensityL2, DensityLinf, PressureL1, PressureL2, PressureLinf) at
# t = 0.2 of the single-level runs whose schemes this library compiles, keyed
# by variant name: (CSV line, norms, blocks of 16 cells). The grids are the
# reference's: 4 nodes of 32 (RK3), 24 or 8 cells, i.e. 128, 96 or 32 cells,
# with the symmetry walls of testsuite/InputFiles/DetailedSod/1D/SodX.xml.
SOD_REFERENCE_NORMS = {
    "fvchar": (58, (6.90089530e-07, 2.05275093e-07, 1.39620303e-07,
                    5.95487513e-07, 2.49384854e-07, 2.28787992e-07), 8),
    "fvchar_weno3_hll": (42, (1.02264424e-06, 2.58609513e-07, 1.78590815e-07,
                              8.47004465e-07, 3.27459497e-07, 2.99812686e-07), 8),
    "fs_weno3": (30, (9.64420466e-07, 2.53172573e-07, 1.78922953e-07,
                      8.43317388e-07, 3.33634664e-07, 3.05663996e-07), 8),
    "fs_llf_weno3": (22, (1.02774396e-06, 2.58481190e-07, 1.81214189e-07,
                          9.21920404e-07, 3.41063398e-07, 3.09256115e-07), 8),
    "fs_llfm_weno3": (74, (9.60803571e-07, 2.56417781e-07, 1.82571444e-07,
                           8.29079300e-07, 3.39286859e-07, 3.11954844e-07), 8),
    "fs_glf_weno5z": (70, (6.11467178e-07, 1.86248795e-07, 1.19883696e-07,
                           5.70962203e-07, 2.28544959e-07, 2.03433021e-07), 8),
    "rk2_fs_glf": (6, (1.79790069e-06, 4.81072783e-07, 2.95788755e-07,
                       1.70715046e-06, 5.93024051e-07, 4.98112838e-07), 6),
    "rk2_fs_llf_weno5z": (10, (4.20347064e-05, 1.71242192e-05, 1.50718666e-05,
                               4.95227518e-05, 2.76342072e-05, 2.66893986e-05), 2),
    "rk2_fvchar_weno3": (34, (2.20465992e-06, 5.65708847e-07, 3.71935085e-07,
                              1.91570490e-06, 6.99942603e-07, 6.14275684e-07), 6),
    "rk2_fvchar_hll_weno5z": (46, (4.18500391e-05, 1.69155498e-05, 1.48248685e-05,
                                   4.66086932e-05, 2.66536675e-05, 2.58109384e-05), 2),
    "rk2_fs_roem_weno3": (50, (2.50746878e-06, 6.35908633e-07, 3.86180985e-07,
                               2.36985780e-06, 8.19966693e-07, 6.63064934e-07), 6),
    "rk2_fs_llfm": (62, (4.73109368e-05, 1.91201415e-05, 1.68388893e-05,
                         5.45096592e-05, 3.08180236e-05, 2.97142519e-05), 2),
    "rk2_fs_llfm_weno5z": (82, (1.28201009e-06, 3.86170496e-07, 1.92486130e-07,
                                1.12651026e-06, 4.31014301e-07, 3.36644260e-07), 6),
    "fs_roem_weno7": (26, (5.41078087e-07, 1.78701534e-07, 1.18724621e-07,
                           4.74130387e-07, 2.22922105e-07, 2.03218512e-07), 8),
    "rk2_fvchar_weno7": (18, (4.53331444e-05, 1.84825089e-05, 1.64356637e-05,
                              5.15861558e-05, 2.92978943e-05, 2.83574250e-05), 2),
    "rk2_fs_glf_weno7": (38, (4.94093395e-05, 1.98145425e-05, 1.74995495e-05,
                              5.98894516e-05, 3.19034136e-05, 3.04606609e-05), 2),
    "rk2_fs_weno7": (54, (1.48258118e-06, 4.43012783e-07, 3.01900864e-07,
                          1.45519660e-06, 5.83116890e-07, 5.16433858e-07), 6),
}


def sod_error_norms(case: cases.Case, u: np.ndarray, t: float) -> np.ndarray:
    """The six DetailedSod norms of a 1D Sod result ``u`` (block layout) at
    time ``t``; the weight is the reference's cell volume, h^3 in 1D too."""
    from oracle.sod_exact import relative_error_norms, sod_exact
    g = case.grid
    glob = g.gather(u)
    rho, energy, mom = glob[0, :, 0, 0], glob[1, :, 0, 0], glob[2, :, 0, 0]
    p = (case.gamma - 1.0) * (energy - 0.5 * mom * mom / rho)
    x = g.cell_centres()[0][:, 0, 0]
    rho_x, _, p_x = sod_exact(x, t, case.gamma)
    vol = g.cell_size ** 3
    return np.concatenate([relative_error_norms(rho, rho_x, vol),
                           relative_error_norms(p, p_x, vol)])


def smooth_bump(c, centre=0.5, radius=0.2):
    """A level case's leaves filled with a pressure and density bump at rest,
    cos^2 in the distance from the centre, zero outside the radius: smooth
    across the level jumps, and uniform at the domain faces."""
    I = cases.interior(c.dim)
    u = c.u.copy()
    for b in range(c.nleaf):
        x = c.cell_centres(b)
        r = np.sqrt(sum((x[d] - centre) ** 2 for d in range(c.dim)))
        w = np.where(r < radius, np.cos(0.5 * np.pi * r / radius) ** 2, 0.0)
        vel = [np.zeros_like(r) for _ in range(c.dim)]
        u[(b, slice(None)) + I[1:]] = cases.primes_to_conservatives(
            c.dim, 1.0 + 0.5 * w, 1.0 + 2.0 * w, vel, c.gamma)
    return u
