"""The fused tile-stage path (alp_engine candidates 4 and 5: one persistent
launch per alp_engine_step call, every block's stage staged into shared memory
by TMA, fluxes and stage update on chip) against the face-flux + stage-update
path (candidate 0), through the C ABI.

The two paths evaluate every 3D face with the same face_compute (the x-face
computation of the rotated stencil, canon_field) and every cell with the same
divergence and stage arithmetic, so the results must be equal bit for bit:
state, time and step count. The face-flux path itself is checked
against the reference in test_gpu_parity.py (and, in the strict build, bit for
bit), and the default 3D engine there now runs the tile path.
"""
import numpy as np
import pytest

import oracle
from alpaca_b200 import api, cases
from alpaca_b200 import native as N

pytestmark = pytest.mark.gpu

FACE, TILE16, TILE12 = 0, 4, 5
I3 = cases.interior(3)


def run(case, variant, cand, precision=N.FP64, strict=False, chunks=(6,), max_steps=None):
    e = api.Engine(3, variant, precision=precision, capacity_blocks=case.grid.nb, max_cases=1,
                   strict=strict)
    e.set_path(cand)
    i = e.add_case(case, max_steps=max_steps)
    for n in chunks:
        e.step(n)
    out = e.get(i)
    assert e.path == cand
    e.close()
    return out


def same(a, b):
    assert np.array_equal(a[0][I3], b[0][I3])
    assert a[1] == b[1] and a[2] == b[2]


@pytest.mark.parametrize("variant", ["fvchar", "fvprim", "fsroe"])
@pytest.mark.parametrize("precision", [N.FP64, N.FP32_FLUX])
def test_tiles_equal_face_path(cuda, variant, precision):
    """3x3x3 periodic Fourier + Mach-2 case, 6 steps, both kernel variants."""
    case = cases.fourier_shock(3, dim=3, seed=41, steps=6)
    ref = run(case, variant, FACE, precision)
    assert ref[2] == 6
    same(run(case, variant, TILE16, precision), ref)
    same(run(case, variant, TILE12, precision), ref)


@pytest.mark.parametrize("periodic", [(0, 0, 0), (cases.SYMMETRY,) * 3,
                                      (1, 0, cases.SYMMETRY), (cases.SYMMETRY, 1, 0)])
def test_tiles_walls(cuda, periodic):
    """Zero-gradient and symmetry walls (no TMA load beyond a wall; the stencil
    maps those cells onto the block) on a 3x2x2 grid with a blast at a corner."""
    g = cases.BlockGrid(3, (3, 2, 2), periodic, 1.0 / 48)
    x, y, z = g.cell_centres()
    r = np.sqrt(x ** 2 + (y - 0.1) ** 2 + (z - 0.05) ** 2)
    rho = np.where(r < 0.2, 2.0, 1.0) + 0.05 * np.sin(7 * x + 3 * y)
    p = np.where(r < 0.2, 8.0, 1.0)
    vel = [0.1 * np.cos(5 * z), -0.2 * np.sin(4 * x), 0.05 + 0 * x]
    glob = cases.primes_to_conservatives(3, rho, p, vel, 1.4)
    case = cases.Case("walls", g, g.scatter(glob), 1.4, 0.0, 0.6, 1e300, 8)
    ref = run(case, "fvchar", FACE)
    same(run(case, "fvchar", TILE16), ref)
    same(run(case, "fvchar", TILE12), ref)


def test_tiles_strict_bit_exact_with_oracle(cuda):
    """Strict build: the tile path reproduces the reference's arithmetic order
    (the oracle) bit for bit over 6 steps, like the face path."""
    case = cases.fourier_shock(2, dim=3, seed=43, steps=6)
    ref = oracle.Restatement(3, "fvchar").run(case.u, case.grid.nbr, case.gamma, 0.0, False,
                                              case.grid.cell_size, case.cfl, 1e300, max_steps=6)
    got = run(case, "fvchar", TILE16, strict=True)
    assert got[2] == 6 and got[1] == ref[1]
    assert np.array_equal(got[0][I3], ref[0][I3])


def test_tiles_steps_across_calls(cuda):
    """Steps split over calls of different lengths (the captured launch's step
    count is updated in place) equal one call; a step budget stops the case."""
    case = cases.fourier_shock(2, dim=3, seed=44, steps=0)
    ref = run(case, "fvchar", FACE, chunks=(10,), max_steps=9)
    assert ref[2] == 9
    same(run(case, "fvchar", TILE16, chunks=(3, 5, 1, 1), max_steps=9), ref)
    same(run(case, "fvchar", TILE16, chunks=(1, 1, 1, 7), max_steps=9), ref)


def test_tiles_rk2(cuda):
    """TVD-RK2 (two stages, stage table entries 3-4) on the tile path."""
    sch = N.Scheme.make("fvchar")
    sch.time_integrator = N.RK2
    case = cases.fourier_shock(2, dim=3, seed=45, steps=5)
    ref = run(case, sch, FACE)
    same(run(case, sch, TILE16), ref)


def test_tiles_multi_case_engine(cuda):
    """Cases of different sizes, materials and end times in one engine: each
    case on the tile path equals the same case alone on the face path; a case
    that reaches its end time mid-call stops exactly there."""
    c1 = cases.fourier_shock(2, dim=3, seed=46, steps=7)
    c2 = cases.water_spheres(2, seed=47)
    c3 = cases.fourier_shock(3, dim=3, seed=48, steps=4)
    alone = [run(c, "fvchar", FACE, chunks=(8,), max_steps=s) for c, s in
             ((c1, 7), (c2, 8), (c3, 4))]
    nb = c1.grid.nb + c2.grid.nb + c3.grid.nb
    e = api.Engine(3, "fvchar", capacity_blocks=nb, max_cases=4)
    assert e.path in (TILE16, TILE12)
    ids = [e.add_case(c1, max_steps=7), e.add_case(c2, max_steps=8), e.add_case(c3, max_steps=4)]
    e.step(5)
    e.step(3)
    got = [e.get(i) for i in ids]
    e.close()
    for a, b in zip(got, alone):
        same(a, b)


def test_tiles_autotune_trials_leave_state(cuda):
    """Trial launches of the tile candidates write scratch pools only and do
    not commit: the case continues exactly as without autotuning."""
    case = cases.fourier_shock(2, dim=3, seed=49, steps=4)
    e = api.Engine(3, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    i = e.add_case(case)
    e.step(2)
    e.autotune(trial_steps=2)
    e.set_path(TILE12)
    e.step(2)
    got = e.get(i)
    e.close()
    same(got, run(case, "fvchar", FACE, chunks=(4,)))


def test_tiles_launch_count(cuda):
    """One step call of the tile path issues three launches whatever its
    length: signal speed, dt and the persistent kernel."""
    case = cases.fourier_shock(2, dim=3, seed=50, steps=0)
    e = api.Engine(3, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    e.add_case(case)
    e.set_path(TILE16)
    assert e.launches(1) == 3 and e.launches(100) == 3
    e.set_path(FACE)
    assert e.launches(10) == 10 * e.launches_per_step
    e.close()
