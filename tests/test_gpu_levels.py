"""Multi-level cases on the GPU (alp_levels_*) against the oracle's restatement
of the same local time stepping.

Tolerances: the strict build reproduces the oracle bit for bit; the fast build
stays within the run tolerance of the single-level tests (per field L1
<= 1e-10 relative) and its micro time steps within 1e-12 relative.
"""
import numpy as np
import pytest

import oracle
from alpaca_b200 import api, cases
from alpaca_b200 import native as N
from helpers import l1_rel, smooth_bump

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-10


def corner(l, lo, hi):
    return all(x == 0 for x in lo)


def corner_tree_with_bump():
    """One refined corner in 3D, with a smooth bump across its level jumps (the
    shock there would make the fifth-order prediction overshoot)."""
    c = cases.spherical_shock_levels(n0=2, dim=3, lmax=2, refine=corner)
    c.u = smooth_bump(c)
    return c


def small_trees():
    return {
        "2d_three_levels": cases.spherical_shock_levels(n0=4, dim=2, lmax=2),
        "3d_corner_three_levels": corner_tree_with_bump(),
        "1d_two_levels": cases.spherical_shock_levels(n0=4, dim=1, lmax=1, nblobs=1,
                                                     refine=lambda l, lo, hi: lo[0] >= 1),
    }


def reference_run(c, variant, macro):
    return oracle.Restatement(c.dim, variant).levels_run(
        c.u, c.level, c.coord, c.n0, c.h0, c.gamma, c.B, False, c.cfl, c.t_end,
        max_macro=macro, nthreads=8)


@pytest.mark.parametrize("name", list(small_trees()))
@pytest.mark.parametrize("variant", ["fvchar", "fsroe"])
def test_levels_match_oracle(cuda, name, variant):
    c = small_trees()[name]
    ref, t_ref, m_ref, dts = reference_run(c, variant, 2)
    eng = api.LevelEngine(c, variant, max_macro=2)
    eng.step(3)  # the third macro step is beyond max_macro: no work
    got, t, m = eng.get()
    info = eng.info()
    eng.close()
    assert m == m_ref == 2
    assert t == pytest.approx(t_ref, rel=1e-12)
    assert info["max_level"] == c.lmax
    I = cases.interior(c.dim)
    for f in range(c.dim + 2):
        assert l1_rel(got[I][:, f], ref[I][:, f]) <= RUN_TOL, (name, f)


@pytest.mark.parametrize("name", ["2d_three_levels", "3d_corner_three_levels"])
@pytest.mark.parametrize("variant", ["fvchar", "fsroe"])
def test_levels_fp32_flux_within_precision_target(cuda, name, variant):
    """The FP32-flux form on multi-level cases (packed FP32 reconstruction,
    FP64 state, ghosts and jump sums in FP64): after two macro steps the
    relative L1 of every field against the FP64 oracle is within the precision
    target 1e-5, and the micro time steps agree to 1e-6."""
    c = small_trees()[name]
    ref, t_ref, m_ref, _ = reference_run(c, variant, 2)
    eng = api.LevelEngine(c, variant, precision=N.FP32_FLUX, max_macro=2)
    eng.step(2)
    got, t, m = eng.get()
    eng.close()
    assert m == m_ref == 2
    assert t == pytest.approx(t_ref, rel=1e-6)
    I = cases.interior(c.dim)
    for f in range(c.dim + 2):
        err = l1_rel(got[I][:, f], ref[I][:, f])
        print(name, variant, "field", f, "fp32 L1", err)
        assert err <= 1e-5, (name, f, err)


@pytest.mark.parametrize("name", ["2d_three_levels", "3d_corner_three_levels"])
def test_levels_strict_bit_exact(cuda, name):
    c = small_trees()[name]
    ref, t_ref, m_ref, _ = reference_run(c, "fvchar", 1)
    eng = api.LevelEngine(c, "fvchar", max_macro=1, strict=True)
    eng.step(1)
    got, t, m = eng.get()
    eng.close()
    I = cases.interior(c.dim)
    assert m == 1 and t == t_ref
    assert np.array_equal(got[I], ref[I])


def test_levels_conserve_mass_and_energy(cuda):
    """Jump-flux correction on the GPU: mass and energy of the 2D three-level
    tree change by round-off only over two macro steps."""
    c = small_trees()["2d_three_levels"]
    eng = api.LevelEngine(c, "fvchar", max_macro=2)
    eng.step(2)
    got, t, m = eng.get()
    eng.close()
    I = cases.interior(2)
    vol = (c.h0 / (1 << c.level)) ** 2

    def tot(u, f):
        return (u[I][:, f].reshape(c.nleaf, -1).sum(1) * vol).sum()

    for f in (0, 1):
        assert abs(tot(got, f) - tot(c.u, f)) <= 1e-14 * tot(c.u, f)


def test_single_level_tree_equals_engine(cuda):
    """A tree without refinement is the single-level engine on the same grid."""
    g = cases.BlockGrid(3, (2, 2, 2), (False,) * 3, 1.0 / 32)
    rng = np.random.default_rng(6)
    x = g.cell_centres()
    shp = g.cells_shape()
    rho = 1 + 0.1 * cases.fourier_modes(rng, shp, x, 3)
    p = 1 + 0.1 * cases.fourier_modes(rng, shp, x, 3)
    vel = [0.2 * cases.fourier_modes(rng, shp, x, 3) for _ in range(3)]
    u = g.scatter(cases.primes_to_conservatives(3, rho, p, vel, 1.4))
    lc = cases.LevelCase("flat", 3, (2, 2, 2), g.cell_size, np.zeros(g.nb, np.int32), g.coords,
                         u, 1.4)
    eng = api.LevelEngine(lc, "fvchar", max_macro=4)
    eng.step(4)
    a, ta, _ = eng.get()
    eng.close()
    flat = cases.Case("flat", g, u, 1.4, 0.0, 0.6, 1e300, 4)
    e2 = api.Engine(3, "fvchar", capacity_blocks=g.nb, max_cases=1)
    cid = e2.add_case(flat, max_steps=4)
    e2.step(4)
    b, tb, steps = e2.get(cid)
    e2.close()
    I = cases.interior(3)
    assert steps == 4 and ta == tb
    assert np.array_equal(a[I], b[I])


def test_spherical_shock_hierarchy_runs(cuda):
    """The 8 / 294 / 1232-leaf hierarchy: one macro step, finite positive
    states, and the launch and work accounting."""
    c = cases.spherical_shock_levels()
    eng = api.LevelEngine(c, "fvchar", max_macro=1)
    info = eng.info()
    eng.step(1)
    got, t, m = eng.get()
    eng.close()
    I = cases.interior(3)
    assert m == 1 and t > 0
    assert np.isfinite(got[I]).all() and (got[I][:, 0] > 0).all()
    assert info["cell_updates_per_macro_step"] == c.cell_updates_per_macro_step()
    assert info["ghosts"] > 0 and info["launches_per_macro_step"] > 0


@pytest.mark.parametrize("variant", ["rk2_fvchar_weno3", "rk2_fs_llf_weno5z", "fvchar_weno7",
                                     "rk2_fvchar_weno7", "fs_glf", "rk2_fs_glf"])
@pytest.mark.parametrize("name", ["2d_three_levels", "3d_corner_three_levels"])
def test_levels_rk2_and_weno7_strict_bit_exact(cuda, name, variant):
    """TVD-RK2 (two stages, jump multipliers 1/2, 1/2), WENO7 (ghosts four
    cells deep) and GlobalLaxFriedrichs (maxima over the leaves computing in
    each stage) on multi-level trees: the strict build against the oracle."""
    c = small_trees()[name]
    ref, t_ref, m_ref, _ = reference_run(c, variant, 1)
    eng = api.LevelEngine(c, variant, max_macro=1, strict=True)
    eng.step(1)
    got, t, m = eng.get()
    eng.close()
    I = cases.interior(c.dim)
    assert m == 1 and t == t_ref
    assert np.isfinite(ref[I]).all()
    assert np.array_equal(got[I], ref[I])


def test_levels_rk2_conserve_mass_and_energy(cuda):
    c = small_trees()["2d_three_levels"]
    eng = api.LevelEngine(c, "rk2_fvchar_weno3", max_macro=2)
    eng.step(2)
    got = eng.get()[0]
    eng.close()
    I = cases.interior(2)
    vol = (c.h0 / (1 << c.level)) ** 2
    for f in (0, 1):
        a = (c.u[I][:, f].reshape(c.nleaf, -1).sum(1) * vol).sum()
        b = (got[I][:, f].reshape(c.nleaf, -1).sum(1) * vol).sum()
        assert abs(b - a) <= 1e-14 * a, f


def test_ghost_wait_runs_out_with_an_error(cuda):
    """The ghost kernel's waits for an earlier group are bounded: when that
    group never finishes (its units are skipped), the waits run out, the step
    ends, and alp_levels_get reports it. The engine's stream and the context
    stay usable, and the next steps run without error again."""
    import torch

    c = cases.spherical_shock_levels(n0=2, dim=3, lmax=2)
    eng = api.LevelEngine(c, "fvchar")
    eng.step(1)
    eng.get()
    assert eng.lib.alp_levels_test_stall_ghosts(eng.h) == N.ALP_OK
    eng.step(1)
    with pytest.raises(N.AlpacaError, match="ran out"):
        eng.get()
    # the error word and counters were cleared: the next step is clean
    eng.step(1)
    _, _, m = eng.get()
    assert m == 3
    x = torch.ones(1 << 20, device="cuda")
    assert float(x.sum()) == float(1 << 20)
    eng.close()
