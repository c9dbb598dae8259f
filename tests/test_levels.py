"""Multi-level cases on the CPU: the oracle's local time stepping reduces to the
single-level loop where it must, and the C ABI rejects trees that are not a
face-balanced tiling before touching the device."""
import ctypes as C

import numpy as np
import pytest

import oracle
from helpers import smooth_bump
from alpaca_b200 import cases
from alpaca_b200 import native as N


def smooth_grid_case(dim, nblocks, cell_size, seed):
    g = cases.BlockGrid(dim, nblocks, (False,) * dim, cell_size)
    rng = np.random.default_rng(seed)
    x = g.cell_centres()
    shp = g.cells_shape()
    rho = 1 + 0.1 * cases.fourier_modes(rng, shp, x, dim)
    p = 1 + 0.1 * cases.fourier_modes(rng, shp, x, dim)
    vel = [0.2 * cases.fourier_modes(rng, shp, x, dim) for _ in range(dim)]
    return g, g.scatter(cases.primes_to_conservatives(dim, rho, p, vel, 1.4))


def test_single_level_tree_is_the_single_level_loop():
    """lmax = 0: one micro step per macro step, same bits as oracle_run."""
    g, u = smooth_grid_case(2, (3, 2), 1.0 / 48, 2)
    R = oracle.Restatement(2, "fvchar")
    a = R.run(u, g.nbr, 1.4, 0.0, False, g.cell_size, 0.6, 1e300, max_steps=3)
    b = R.levels_run(u, np.zeros(g.nb, np.int32), g.coords, (3, 2), g.cell_size, 1.4, 0.0, False,
                     0.6, 1e300, max_macro=3)
    I = cases.interior(2)
    assert np.array_equal(a[0][I], b[0][I])
    assert a[1] == b[1] and np.array_equal(a[3], b[3])


def test_uniform_finer_level_takes_two_micro_steps():
    """All leaves on level 1: two micro steps per macro step, each the
    single-level step with the level-1 cell size (final time may differ in the
    last bit: the macro time adds the micro steps as one sum)."""
    g, u = smooth_grid_case(2, (4, 2), 1.0 / 64, 3)
    R = oracle.Restatement(2, "fsroe")
    a = R.run(u, g.nbr, 1.4, 0.0, False, g.cell_size, 0.6, 1e300, max_steps=4)
    b = R.levels_run(u, np.ones(g.nb, np.int32), g.coords, (2, 1), 2 * g.cell_size, 1.4, 0.0,
                     False, 0.6, 1e300, max_macro=2)
    I = cases.interior(2)
    assert np.array_equal(a[0][I], b[0][I])
    assert np.array_equal(a[3], b[3]) and abs(a[1] - b[1]) <= 1e-15 * a[1]


def totals(c, u):
    I = cases.interior(c.dim)
    vol = (c.h0 / (1 << c.level)) ** c.dim
    return np.array([(u[I][:, f].reshape(c.nleaf, -1).sum(1) * vol).sum()
                     for f in range(c.dim + 2)])


def corner(l, lo, hi):
    return all(x == 0 for x in lo)


@pytest.mark.parametrize("dim,macro", [(1, 2), (2, 2), (3, 1)])
def test_three_level_tree_conserves_mass_and_energy(dim, macro):
    """Three-level trees with the jump-flux correction: mass and energy are
    conserved to round-off while no wave reaches the domain faces (without the
    correction the 2D tree loses 1.7e-8 of its mass per macro step)."""
    if dim == 1:
        c = cases.spherical_shock_levels(n0=4, dim=1, lmax=2, nblobs=1)
    elif dim == 2:
        c = cases.spherical_shock_levels(n0=4, dim=2, lmax=2)
    else:
        # one refined corner, with a smooth bump across its level jumps (a
        # shock there would make the fifth-order prediction overshoot)
        c = cases.spherical_shock_levels(n0=2, dim=3, lmax=2, refine=corner)
        c.u = smooth_bump(c)
    u, t, m, dts = oracle.Restatement(dim, "fvchar").levels_run(
        c.u, c.level, c.coord, c.n0, c.h0, c.gamma, 0.0, False, 0.6, 1e300, max_macro=macro,
        nthreads=4)
    I = cases.interior(dim)
    assert m == macro and len(dts) == 4 * macro and np.all(dts > 0)
    assert t == pytest.approx(dts.sum())
    assert np.isfinite(u[I]).all() and (u[I][:, 0] > 0).all()
    a, b = totals(c, c.u), totals(c, u)
    assert abs(b[0] - a[0]) <= 1e-14 * a[0] and abs(b[1] - a[1]) <= 1e-14 * a[1]


def test_rk2_three_level_tree_conserves_mass_and_energy():
    """TVD-RK2 on a three-level 2D tree: jump multipliers 1/2, 1/2 keep the
    jump-flux correction exact."""
    c = cases.spherical_shock_levels(n0=4, dim=2, lmax=2)
    u, t, m, dts = oracle.Restatement(2, "rk2_fvchar_weno3").levels_run(
        c.u, c.level, c.coord, c.n0, c.h0, c.gamma, 0.0, False, 0.6, 1e300, max_macro=2,
        nthreads=4)
    I = cases.interior(2)
    assert m == 2 and np.isfinite(u[I]).all()
    a, b = totals(c, c.u), totals(c, u)
    assert abs(b[0] - a[0]) <= 1e-14 * a[0] and abs(b[1] - a[1]) <= 1e-14 * a[1]


def test_leaves_per_level_of_the_spherical_shock_hierarchy():
    c = cases.spherical_shock_levels()
    assert c.leaves_per_level() == [8, 294, 1232]
    assert c.cell_updates_per_macro_step() == 4096 * (8 + 2 * 294 + 4 * 1232)


# ---- the C ABI validates the tree on the host --------------------------------

def _create(dim, n0, level, coord, h0=1.0 / 32):
    lib = N.lib()
    sch = N.Scheme.make("fvchar")
    mat = N.Material.make(1.4)
    level = np.ascontiguousarray(level, dtype=np.int32)
    coord = np.ascontiguousarray(coord, dtype=np.int32).reshape(-1, 3)
    n0 = np.ascontiguousarray(list(n0) + [1] * (3 - len(n0)), dtype=np.int32)
    u = np.zeros((len(level), dim + 2) + cases.block_shape(dim))
    h = C.c_void_p()
    rc = lib.alp_levels_create(dim, C.byref(sch), C.byref(mat), n0.ctypes.data_as(N._I), h0,
                               len(level), level.ctypes.data_as(N._I),
                               coord.ctypes.data_as(N._I), 0.6, 0.0, 1.0, 1,
                               u.ctypes.data_as(N._D), C.byref(h))
    return rc, lib.alp_last_error().decode()


@pytest.mark.parametrize("what", ["overlap", "gap", "unbalanced", "level", "outside"])
def test_invalid_trees_are_rejected(what):
    if what == "overlap":  # a leaf and its parent
        rc, msg = _create(1, (2,), [0, 0, 1, 1], [[0, 0, 0], [1, 0, 0], [0, 0, 0], [1, 0, 0]])
    elif what == "gap":  # level-0 node 1 missing
        rc, msg = _create(1, (2,), [0], [[0, 0, 0]])
    elif what == "unbalanced":  # level-2 leaves next to a level-0 leaf
        lv = [0, 1, 2, 2]
        co = [[1, 0, 0], [0, 0, 0], [2, 0, 0], [3, 0, 0]]
        rc, msg = _create(1, (2,), lv, co)
        assert "more than one level" in msg
    elif what == "level":
        rc, msg = _create(1, (1,), [9], [[0, 0, 0]])
    else:
        rc, msg = _create(1, (2,), [0, 0], [[0, 0, 0], [2, 0, 0]])
    assert rc == N.ALP_ERR_INVALID, (what, rc, msg)
    assert msg


def test_global_lax_friedrichs_three_level_tree_conserves():
    """GlobalLaxFriedrichs on a three-level tree: the wave speeds are the maxima
    over the leaves computing in each stage (as ComputeRightHandSide takes
    them over the levels it is given); mass and energy stay conserved. No
    density blobs: their tails reach the zero-gradient domain faces, where the
    global wave speed's dissipation moves mass through the faces (6e-9 of it
    in two macro steps on a single level too)."""
    c = cases.spherical_shock_levels(n0=4, dim=2, lmax=2, nblobs=0)
    u, t, m, dts = oracle.Restatement(2, "fs_glf").levels_run(
        c.u, c.level, c.coord, c.n0, c.h0, c.gamma, 0.0, False, 0.6, 1e300, max_macro=2,
        nthreads=4)
    I = cases.interior(2)
    assert m == 2 and np.isfinite(u[I]).all()
    a, b = totals(c, c.u), totals(c, u)
    assert abs(b[0] - a[0]) <= 1e-14 * a[0] and abs(b[1] - a[1]) <= 1e-14 * a[1]
