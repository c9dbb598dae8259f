"""The 1D Sod shock tube against its exact solution, scored the way the
reference testsuite scores its DetailedSod case, and pinned to the error table
the reference recorded from its own runs.

The grid is the reference's: [0, 1] in 128 cells (here 8 blocks of 16, there
4 blocks of 32: the single-level scheme does not see block boundaries), CFL
0.6, t_end 0.2, zero-gradient ends. The table holds 9 significant digits, so
the oracle's norms agree with it to <= 1e-8 relative.
"""
import numpy as np
import pytest

import oracle
from alpaca_b200 import cases
from helpers import SOD_REFERENCE_NORMS, sod_error_norms
from oracle.sod_exact import sod_exact

TABLE_TOL = 1e-8


def test_exact_solution_star_state():
    """Star region of the Sod problem as tabulated by Toro (test 1, table 4.2:
    p* = 0.30313, u* = 0.92745, rho*L = 0.42632, rho*R = 0.26557)."""
    x = np.array([0.55, 0.75])  # left and right of the contact at t = 0.2
    rho, vel, p = sod_exact(x, 0.2)
    assert p == pytest.approx([0.30313, 0.30313], abs=1e-5)
    assert vel == pytest.approx([0.92745, 0.92745], abs=1e-5)
    assert rho == pytest.approx([0.42632, 0.26557], abs=1e-5)


def test_exact_solution_shock_jump_conditions():
    """Mass and momentum fluxes are continuous across the right shock in its
    frame."""
    g = 1.4
    rho, vel, p = sod_exact(np.array([0.85, 0.9]), 0.2)
    rr, ur, pr = 0.125, 0.0, 0.1
    s = (rho[0] * vel[0] - rr * ur) / (rho[0] - rr)  # mass flux continuity
    assert 0.85 < 0.5 + s * 0.2 < 0.9
    m_l = rho[0] * (vel[0] - s)
    assert m_l * (vel[0] - s) + p[0] == pytest.approx(rr * (ur - s) ** 2 + pr, rel=1e-12)
    e_l = p[0] / (g - 1) / rho[0] + 0.5 * (vel[0] - s) ** 2 + p[0] / rho[0]
    e_r = pr / (g - 1) / rr + 0.5 * (ur - s) ** 2 + pr / rr
    assert e_l == pytest.approx(e_r, rel=1e-12)


@pytest.mark.parametrize("variant", list(SOD_REFERENCE_NORMS))
def test_oracle_sod_norms_match_reference_table(variant):
    line, ref = SOD_REFERENCE_NORMS[variant]
    case = cases.sod_1d()
    u, t, steps, _ = oracle.Restatement(1, variant).run(
        case.u, case.grid.nbr, case.gamma, 0.0, False, case.grid.cell_size, case.cfl,
        case.t_end)
    assert t == case.t_end and steps == 92
    got = sod_error_norms(case, u, t)
    assert np.max(np.abs(got / np.array(ref) - 1.0)) <= TABLE_TOL, (variant, line, got)
