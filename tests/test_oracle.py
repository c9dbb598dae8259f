"""The CPU oracle, pinned three ways (no GPU needed):

1. known-answer values from the reference's own unit tests,
2. bit-for-bit agreement with the reference's sources compiled by oracle/Makefile
   (skipped where oracle/_ref was not built),
3. the committed golden fixtures generated from those reference builds.
"""
import glob
import hashlib
import os

import numpy as np
import pytest

import oracle
from alpaca_b200 import cases
from helpers import filled, small_cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EPS = np.finfo(np.float64).eps


def approx_eps(value, expected, eps=EPS):
    # Catch2 Approx(expected).epsilon(eps): |v - e| <= eps * (scale + max(|v|, |e|)), scale 0
    return abs(value - expected) <= eps * max(abs(value), abs(expected))


def approx_margin(value, expected, margin):
    # Catch2 Approx(expected).margin(m) keeps the default epsilon 100 * FLT_EPSILON
    return abs(value - expected) <= margin or approx_eps(value, expected,
                                                         100 * np.finfo(np.float32).eps)


# ---- 1. reference unit-test values ------------------------------------------

def test_weno5_unity_and_step():
    """test/stencils/test_stencils.cpp:137-153 (WENO5: unity 1e-16, step 1e-11)."""
    R = oracle.Restatement(3)
    l, r = R.weno5(np.ones(6))
    assert abs(l - 1.0) <= 1e-16 and abs(r - 1.0) <= 1e-16
    l, r = R.weno5(np.array([0, 0, 0, 1, 1, 1.0]))
    assert abs(l - 0.0) <= 1e-11 and abs(r - 1.0) <= 1e-11


ARB_CONS = np.array([1.2, 4.5, 0.36, 2.7, 3.05])     # mass, energy, mx, my, mz
ARB_PRIM = np.array([2.4, 3.75, 0.75, 1.9, 4.003])   # rho, p, u, v, w


def test_stiffened_gas_known_answers():
    """test/materials/test_equations_of_state.cpp:157-184 (gamma 1.6, B 2)."""
    out = oracle.Restatement(3).eos(1.6, 2.0, False, ARB_CONS, ARB_PRIM)
    assert approx_eps(out[0], -4.6805249999999994)
    assert approx_eps(out[1], -0.1504374999999995)
    assert approx_eps(out[2], 35.819144133333332)
    assert approx_eps(out[3], 1.957890020745122)
    assert approx_eps(out[4], 2.8958333333333335)
    assert approx_eps(out[5], 0.6)


def test_stiffened_gas_safe_known_answers():
    """test/materials/test_equations_of_state.cpp:214-237 (safe, gamma 1.2, B 0.2)."""
    out = oracle.Restatement(3).eos(1.2, 0.2, True, ARB_CONS, ARB_PRIM)
    assert approx_eps(out[0], -0.19999999999999979)
    assert approx_eps(out[1], 3.5833333333333335)
    assert approx_eps(out[2], 44.185810800000006)
    assert approx_eps(out[3], 1.4053469322555197)
    assert approx_eps(out[4], 1.6625000000000001)


def test_generic_stiffened_gas():
    """test/materials/test_generic_stiffened_gas.cpp:76-136."""
    R = oracle.Restatement(3)
    # CalculateEnergy(1.1, 0.1, 0.2, 0.3, 2.0, 1.4, 3.0) = 15.577
    e = R.eos(1.4, 3.0, False, np.ones(5), np.array([1.1, 2.0, 0.1, 0.2, 0.3]))[2]
    assert approx_margin(e, 15.577, 1e-15)
    # pressure with zero density: safe > 0, unsafe not a normal number
    cons = np.array([0.0, 2.0, 0.1, 0.2, 0.3])
    with np.errstate(all="ignore"):
        assert R.eos(1.4, 0.0, True, cons, np.ones(5))[0] > 0.0
        p = R.eos(1.4, 0.0, False, cons, np.ones(5))[0]
    assert not np.isfinite(p) or p == 0.0 or abs(p) < np.finfo(float).tiny
    # speed of sound of p = -1e-4, B = 0: safe > 0, unsafe NaN
    prim = np.array([1.0, -0.0001, 0.0, 0.0, 0.0])
    assert R.eos(1.4, 0.0, True, np.ones(5), prim)[3] > 0.0
    assert np.isnan(R.eos(1.4, 0.0, False, np.ones(5), prim)[3])


def test_prime_state_round_trip():
    """test/prime_states/test_prime_state_handler.cpp:76-140: primes (2..6) ->
    conservatives -> primes, gamma 1.4, B 1."""
    for dim in (1, 2, 3):
        R = oracle.Restatement(dim)
        ne = dim + 2
        shp = (1, ne) + cases.block_shape(dim)
        prim = np.arange(2.0, 2.0 + ne)
        rho, p, vel = prim[0], prim[1], list(prim[2:])
        cons = cases.primes_to_conservatives(dim, np.array(rho), np.array(p),
                                             [np.array(v) for v in vel], 1.4, 1.0)
        u = np.broadcast_to(cons.reshape((1, ne, 1, 1, 1)), shp).copy()
        back = R.prime_states(u, 1.4, 1.0, False)[0, :, 0, 0, 0]
        assert np.allclose(back, prim, rtol=1e-13, atol=0)


def test_halo_known_answer():
    """test/communication/test_internal_halo_manager.cpp:76-140: 2x2x2 blocks
    each filled with its id; after the update every halo region holds the id
    of the neighbour in that direction."""
    g = cases.BlockGrid(3, (2, 2, 2), (False, False, False), 1.0 / 32)
    u = np.zeros((g.nb, 1) + cases.block_shape(3))
    for b in range(g.nb):
        u[b] = b
    oracle.Restatement(3).halo_fill(u, g.nbr26)
    checked = 0
    for b in range(g.nb):
        for s in range(26):
            o = s if s < 13 else s + 1
            off = (o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1)
            n = g.nbr26[b, s]
            sl = tuple(slice(20, 24) if x > 0 else slice(0, 4) if x < 0 else slice(4, 20)
                       for x in off)
            region = u[(b, 0) + sl]
            if n >= 0:
                assert np.all(region == n), (b, off)
                checked += 1
            else:  # domain side: untouched, still the block's own id
                assert np.all(region == b)
    assert checked == 8 * 7  # each block has 7 neighbours in a 2x2x2 box


# ---- 2. bit-for-bit against the compiled reference ----------------------------

needs_ref = pytest.mark.skipif(not oracle.Reference.available(),
                               reason="oracle/_ref not built (reference sources absent)")


@needs_ref
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("variant", list(oracle.VARIANTS))
def test_restatement_matches_reference_rhs(dim, variant):
    case = small_cases()[dim]
    u = filled(case)
    a = oracle.Restatement(dim, variant).space_rhs(u, case.gamma, 0.0, False, case.grid.cell_size)
    b = oracle.Reference(dim, variant).space_rhs(u, case.gamma, 0.0, False, case.grid.cell_size)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@needs_ref
@pytest.mark.parametrize("variant", list(oracle.VARIANTS))
def test_restatement_matches_reference_stiffened(variant):
    """Stiffened gas (water-like gamma 6.12, B 3000 in non-dimensional units) and
    the safe EOS variant, 3D, one block."""
    case = cases.fourier_shock(1, dim=3, seed=11, gamma=6.12, B=3000.0)
    u = filled(case)
    for safe in (False, True):
        a = oracle.Restatement(3, variant).space_rhs(u, 6.12, 3000.0, safe, case.grid.cell_size)
        b = oracle.Reference(3, variant).space_rhs(u, 6.12, 3000.0, safe, case.grid.cell_size)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@needs_ref
@pytest.mark.parametrize("variant", list(oracle.VARIANTS))
def test_restatement_matches_reference_run(variant):
    case = cases.sod_1d()
    a = oracle.Restatement(1, variant).run(case.u, case.grid.nbr, 1.4, 0.0, False,
                                           case.grid.cell_size, 0.6, 0.2)
    b = oracle.Reference(1, variant).run(case.u, case.grid.nbr, 1.4, 0.0, False,
                                         case.grid.cell_size, 0.6, 0.2)
    I = cases.interior(1)
    assert np.array_equal(a[0][I], b[0][I])
    assert a[1] == b[1] and a[2] == b[2] and np.array_equal(a[3], b[3])


# ---- 3. committed golden fixtures ---------------------------------------------

def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "rhs_d*.npz"))),
                         ids=os.path.basename)
def test_restatement_matches_golden_rhs(path):
    z = np.load(path)
    name = os.path.basename(path)[:-4]
    dim = int(name.split("_")[1][1])
    variant = name.split("_")[2]
    case = small_cases()[dim]
    u = filled(case)
    assert _sha(u) == str(z["input_sha"]), "case generator no longer reproduces the fixture input"
    rhs = oracle.Restatement(dim, variant).space_rhs(u, case.gamma, 0.0, False,
                                                     case.grid.cell_size)[3]
    assert np.array_equal(rhs[cases.interior(dim)], z["rhs"])
    dt = oracle.Restatement(dim).timestep(u, case.gamma, 0.0, False, case.grid.cell_size, case.cfl)
    assert dt == float(z["dt"])


@pytest.mark.parametrize("variant", list(oracle.VARIANTS))
def test_restatement_matches_golden_sod(variant):
    z = np.load(os.path.join(GOLDEN, f"sod1d_{variant}.npz"))
    case = cases.sod_1d()
    assert _sha(case.u) == str(z["input_sha"])
    u, t, steps, dts = oracle.Restatement(1, variant).run(case.u, case.grid.nbr, 1.4, 0.0, False,
                                                          case.grid.cell_size, 0.6, 0.2)
    assert steps == int(z["steps"]) and t == float(z["t"])
    assert np.array_equal(dts, z["dts"])
    assert np.array_equal(u[cases.interior(1)], z["final"])


def test_sod_physics_sanity():
    """Sod at t = 0.2 from the fixture: density between the initial states,
    contact/shock structure monotone where the exact solution is."""
    z = np.load(os.path.join(GOLDEN, "sod1d_fvchar.npz"))
    rho = z["final"][:, 0].reshape(-1)
    assert abs(float(z["t"]) - 0.2) < 1e-15
    assert rho.min() > 0.124 and rho.max() < 1.001  # WENO over/undershoots stay small
    assert rho[0] == pytest.approx(1.0, abs=1e-6) and rho[-1] == pytest.approx(0.125, abs=1e-6)


# ---- 4. operation counts (the FP64 compute ceiling of the path) --------------

@pytest.mark.parametrize("dim", [2, 3])
def test_op_counts_match_bench_constants(dim):
    """The operation-counting build computes the restatement's results bit for
    bit, and its flops per 2D / 3D cell-update are the constants bench.py
    reports (the 2D ones bound the serving streams' makespan)."""
    import bench
    case = cases.fourier_shock(1, dim=dim, seed=5)
    u = filled(case)
    table = bench.FLOPS_PER_CELL_UPDATE_3D if dim == 3 else bench.FLOPS_PER_CELL_UPDATE_2D
    for variant, expected in table.items():
        O = oracle.OpCounting(dim, variant)
        a = oracle.Restatement(dim, variant).space_rhs(u, case.gamma, 0.0, False,
                                                       case.grid.cell_size)[3]
        b = O.space_rhs(u, case.gamma, 0.0, False, case.grid.cell_size)[3]
        assert np.array_equal(a, b)
        O.reset()
        O.run(case.u, case.grid.nbr, case.gamma, 0.0, False, case.grid.cell_size, case.cfl,
              1e300, max_steps=1)
        c = O.counts()
        flops = (c["add"] + c["mul"] + c["div"] + c["sqrt"]) / 16 ** dim
        assert abs(flops - expected) <= 0.01 * expected, (variant, flops)


# ---- 5. further selections: stencils, Riemann solvers, signal speeds, splittings

EXT = list(oracle.EXT_VARIANTS)


@pytest.mark.parametrize("dim", [1, 3])
@pytest.mark.parametrize("variant", EXT)
def test_ext_restatement_matches_reference_rhs(dim, variant):
    if not oracle.Reference.available(dim, variant):
        pytest.skip("oracle/_ref further selections not built (make -C oracle ref-ext)")
    case = small_cases()[dim]
    u = filled(case)
    a = oracle.Restatement(dim, variant).space_rhs(u, case.gamma, 0.0, False, case.grid.cell_size)
    b = oracle.Reference(dim, variant).space_rhs(u, case.gamma, 0.0, False, case.grid.cell_size)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("variant", EXT)
def test_ext_restatement_matches_golden(variant):
    """RHS in 1D and 3D and the 1D Sod run to t = 0.2, from the reference."""
    for dim in (1, 3):
        z = np.load(os.path.join(GOLDEN, "ext", f"rhs_d{dim}_{variant}.npz"))
        case = small_cases()[dim]
        u = filled(case)
        assert _sha(u) == str(z["input_sha"])
        rhs = oracle.Restatement(dim, variant).space_rhs(u, case.gamma, 0.0, False,
                                                         case.grid.cell_size)[3]
        assert np.array_equal(rhs[cases.interior(dim)], z["rhs"])
    z = np.load(os.path.join(GOLDEN, "ext", f"sod1d_{variant}.npz"))
    case = cases.sod_1d()
    u, t, steps, dts = oracle.Restatement(1, variant).run(case.u, case.grid.nbr, 1.4, 0.0, False,
                                                          case.grid.cell_size, 0.6, 0.2)
    assert steps == int(z["steps"]) and t == float(z["t"]) and np.array_equal(dts, z["dts"])
    assert np.array_equal(u[cases.interior(1)], z["final"])


@pytest.mark.parametrize("variant", EXT)
def test_ext_selection_changes_the_scheme(variant):
    base = oracle.EXT_VARIANTS[variant][0]
    case = small_cases()[3]
    u = filled(case)
    a = oracle.Restatement(3, variant).space_rhs(u, case.gamma, 0.0, False, case.grid.cell_size)[3]
    b = oracle.Restatement(3, base).space_rhs(u, case.gamma, 0.0, False, case.grid.cell_size)[3]
    assert not np.array_equal(a, b)
