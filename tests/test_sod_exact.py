"""The 1D Sod shock tube against its exact solution, scored the way the
reference testsuite scores its DetailedSod case, and pinned to the error table
the reference recorded from its own runs.

The grids are the reference's: [0, 1] in 128, 96 or 32 cells (here blocks of
16, there 4 nodes of 32, 24 or 8: the single-level scheme does not see block
boundaries), symmetry walls at both ends as SodX.xml sets them, CFL 0.6,
t_end 0.2; SSP-RK3 and TVD-RK2 rows. The table holds 9 significant digits, so
the oracle's norms agree with it to <= 1e-8 relative. (With zero-gradient ends
instead, the 32-cell rows of the more dissipative schemes move by up to 7e-6:
their shock profile reaches the wall's stencil.)
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
    line, ref, nblocks = SOD_REFERENCE_NORMS[variant]
    case = cases.sod_1d(nblocks, symmetry=True)
    u, t, steps, _ = oracle.Restatement(1, variant).run(
        case.u, case.grid.nbr, case.gamma, 0.0, False, case.grid.cell_size, case.cfl,
        case.t_end)
    assert t == case.t_end
    got = sod_error_norms(case, u, t)
    assert np.max(np.abs(got / np.array(ref) - 1.0)) <= TABLE_TOL, (variant, line, got)


@pytest.mark.parametrize("variant", ["fs_glf_weno5z", "rk2_fs_llfm", "rk2_fvchar_weno3"])
def test_symmetry_walls_restatement_is_the_reference(variant):
    """The symmetry-wall halos and the RK2 loop of the restatement against the
    reference's compiled code (SymmetryInternalValue / RungeKutta2TVD), bit
    for bit over the whole run."""
    if not oracle.Reference.available(1, variant):
        pytest.skip("oracle/_ref further selections not built (make -C oracle ref-ext)")
    _, _, nblocks = SOD_REFERENCE_NORMS[variant]
    case = cases.sod_1d(nblocks, symmetry=True)
    args = (case.u, case.grid.nbr, case.gamma, 0.0, False, case.grid.cell_size, case.cfl,
            case.t_end)
    a = oracle.Restatement(1, variant).run(*args)
    b = oracle.Reference(1, variant).run(*args)
    assert a[2] == b[2] and a[1] == b[1] and np.array_equal(a[0], b[0])


def test_symmetry_walls_in_the_grid():
    g = cases.BlockGrid(2, (2, 3), (cases.SYMMETRY, True), 0.1)
    # x walls on face slots only, y periodic
    assert (g.nbr[:, 0] == -2).sum() == 3 and (g.nbr[:, 1] == -2).sum() == 3
    assert (g.nbr[:, 2] >= 0).all() and (g.nbr[:, 3] >= 0).all()
    assert not (np.delete(g.nbr26, [4, 21], axis=1) == -2).any()
