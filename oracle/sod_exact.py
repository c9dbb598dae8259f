"""Exact Sod shock-tube solution and the reference's relative error norms
(TEST INFRASTRUCTURE ONLY: the checker of shock-tube runs, never shipped).

The reference scores its DetailedSod test case
(python/alpacapy/testsuite/test_cases/detailed_sod.py:87) with
``SodAnalysis.compare_to_exact_solution``
(python/alpacapy/post_analysis/sod_analysis.py:240-279): the exact Riemann
solution at the cell centres (sod_analysis.py:109-200, membrane at x = 0.5) and
``compute_relative_error_norms`` (python/alpacapy/helper_functions/
mathematical_operations.py:25-51) of density and pressure with the cell volume
as weight.

The exact solution here is the textbook one (Toro, "Riemann Solvers and
Numerical Methods for Fluid Dynamics", ch. 4): the star pressure from Newton's
method on the pressure function, a left rarefaction, a contact and a right
shock. The reference iterates on the shock Mach number instead; both solve the
same equations, so the states agree to round-off.
"""
from __future__ import annotations

import numpy as np


def _pressure_function(p, rho_k, p_k, c_k, g):
    """Velocity jump across the left/right wave and its derivative in p."""
    if p > p_k:  # shock
        a = 2.0 / ((g + 1.0) * rho_k)
        b = (g - 1.0) / (g + 1.0) * p_k
        q = np.sqrt(a / (p + b))
        return (p - p_k) * q, q * (1.0 - 0.5 * (p - p_k) / (b + p))
    r = (p / p_k) ** ((g - 1.0) / (2.0 * g))  # rarefaction
    return 2.0 * c_k / (g - 1.0) * (r - 1.0), r / (rho_k * c_k) * (p_k / p)


def sod_exact(x, t, gamma=1.4, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1), x0=0.5):
    """Density, velocity and pressure at positions ``x`` and time ``t`` of a
    Riemann problem whose star region holds a left rarefaction and a right
    shock (the Sod configuration)."""
    g = gamma
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    p = 0.5 * (pl + pr)
    for _ in range(100):
        fl, dl = _pressure_function(p, rl, pl, cl, g)
        fr, dr = _pressure_function(p, rr, pr, cr, g)
        step = (fl + fr + ur - ul) / (dl + dr)
        p -= step
        if abs(step) <= 1e-15 * p:
            break
    fl, _ = _pressure_function(p, rl, pl, cl, g)
    fr, _ = _pressure_function(p, rr, pr, cr, g)
    if not (p > pr and p < pl):
        raise ValueError("not a rarefaction-contact-shock configuration")
    us = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    rho_ls = rl * (p / pl) ** (1.0 / g)
    mu = (g - 1.0) / (g + 1.0)
    rho_rs = rr * (p / pr + mu) / (mu * p / pr + 1.0)
    c_ls = cl * (p / pl) ** ((g - 1.0) / (2.0 * g))
    s_shock = ur + cr * np.sqrt((g + 1.0) / (2.0 * g) * p / pr + (g - 1.0) / (2.0 * g))
    xi = (np.asarray(x, dtype=np.float64) - x0) / t
    head, tail = ul - cl, us - c_ls
    fan = 2.0 / (g + 1.0) + mu / cl * (ul - xi)
    rho = np.select([xi < head, xi < tail, xi < us, xi < s_shock],
                    [rl, rl * fan ** (2.0 / (g - 1.0)), rho_ls, rho_rs], rr)
    vel = np.select([xi < head, xi < tail, xi < s_shock],
                    [ul, 2.0 / (g + 1.0) * (cl + 0.5 * (g - 1.0) * ul + xi), us], ur)
    pres = np.select([xi < head, xi < tail, xi < s_shock],
                     [pl, pl * fan ** (2.0 * g / (g - 1.0)), p], pr)
    return rho, vel, pres


def relative_error_norms(solution, exact, cell_volume):
    """(L1, L2, Linf) of |solution / exact - 1| weighted by the cell volume,
    as mathematical_operations.py:49-51 defines them."""
    e = np.abs(np.asarray(solution) / np.asarray(exact) - 1.0) * cell_volume
    return np.array([e.sum(), np.sqrt((e * e).sum()), e.max()])
