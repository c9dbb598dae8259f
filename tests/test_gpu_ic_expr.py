"""Initial conditions given as expressions, evaluated on the device
(alp_ic_evaluate, alp_engine_add_case_expr), against the oracle's evaluation
of the same programs.

Tolerance: per prime state max|d| <= 1e-13 max|ref|. CUDA's and the host's
transcendental functions may differ in the last bits; everything else is the
same arithmetic in the same order.
"""
import numpy as np
import pytest
import torch

from alpaca_b200 import api, cases
from alpaca_b200 import native as N
from helpers import SOD_REFERENCE_NORMS, sod_error_norms
from oracle import ic_expr as X
from test_ic_expr import PROGRAMS, SOD

pytestmark = pytest.mark.gpu

TOL = 1e-13


def close(got, ref):
    for f in range(ref.shape[1]):
        r, g = ref[:, f], got[:, f]
        scale = max(np.nanmax(np.abs(r)), 1e-300)
        assert np.array_equal(np.isnan(g), np.isnan(r)), f
        ok = ~np.isnan(r)
        assert np.max(np.abs(g[ok] - r[ok]), initial=0.0) <= TOL * scale, f


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("name", list(PROGRAMS))
def test_device_prime_states_match_oracle(cuda, dim, name):
    rng = np.random.default_rng(dim)
    nb = 3
    h = 0.7 / 16
    origins = np.zeros((nb, 3))
    origins[:, :dim] = rng.uniform(-0.1, 0.6, (nb, dim))
    units = (2.0, 0.5, 1.5)
    prog = api.IcProgram(PROGRAMS[name])
    got = prog.evaluate(torch.from_numpy(origins).to(cuda), dim, h / units[2],
                        units=N.Units(*units)).cpu().numpy()
    prog.close()
    ref = X.initial_prime_states(PROGRAMS[name], dim, origins, h, units=units)
    close(got, ref)


def test_engine_sod_from_expression_meets_reference_table(cuda):
    """The Sod program of the reference's DetailedSod input, evaluated on the
    device into an engine case with its symmetry walls, run to t = 0.2: the
    reference's error table."""
    case = cases.sod_1d()
    prog = api.IcProgram(SOD)
    eng = api.Engine(1, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    cid = eng.add_case_expr(prog, (case.grid.nb,), case.grid.cell_size,
                            N.Material.make(case.gamma), periodic=(cases.SYMMETRY, 0, 0),
                            cfl=case.cfl, t_end=case.t_end)
    u0 = eng.get(cid)[0]
    I = cases.interior(1)
    np.testing.assert_allclose(u0[I], case.u[I], rtol=1e-15, atol=0)
    eng.run_to_end(chunk=50)
    u, t, steps = eng.get(cid)
    eng.close()
    prog.close()
    assert steps == 92
    got = sod_error_norms(case, u, t)
    assert np.max(np.abs(got / np.array(SOD_REFERENCE_NORMS["fvchar"][1]) - 1)) <= 1e-7


def test_engine_expression_case_matches_array_case(cuda):
    """A smooth 3D program on 2x2x2 blocks: the engine case made on the device
    and the same initial state uploaded from the oracle agree after 5 steps."""
    text = """density := 1 + 0.1 sin(2 * pi * x) cos(2 * pi * y);
              velocityX := 0.2 cos(2 * pi * z); velocityY := 0.1;
              velocityZ := -0.1 sin(2 * pi * x); pressure := 1 + 0.1 * cos(2 * pi * (x + y + z));"""
    g = cases.BlockGrid(3, (2, 2, 2), (True,) * 3, 1.0 / 32)
    prims = X.initial_prime_states(text, 3, np.array(g.coords) * 16 * g.cell_size, g.cell_size)
    u = np.zeros((g.nb, 5) + cases.block_shape(3))
    I = cases.interior(3)
    rho, p, vel = prims[:, 0], prims[:, 1], [prims[:, 2], prims[:, 3], prims[:, 4]]
    cons = cases.primes_to_conservatives(3, rho, p, vel, 1.4)
    u[I] = np.moveaxis(np.asarray(cons), 0, 1).reshape((g.nb, 5, 16, 16, 16))
    mat = N.Material.make(1.4)
    prog = api.IcProgram(text)
    eng = api.Engine(3, "fvchar", capacity_blocks=2 * g.nb, max_cases=2)
    a = eng.add_case_expr(prog, (2, 2, 2), g.cell_size, mat, periodic=(1, 1, 1), max_steps=5)
    b = eng.add_case(cases.Case("arr", g, u, 1.4, 0.0, 0.6, 1e300, 5), max_steps=5)
    eng.step(5)
    ua, ta, _ = eng.get(a)
    ub, tb, _ = eng.get(b)
    eng.close()
    prog.close()
    assert ta == pytest.approx(tb, rel=1e-14)
    for f in range(5):
        assert np.abs(ua[I][:, f] - ub[I][:, f]).max() <= 1e-13 * np.abs(ub[I][:, f]).max()


def test_expression_case_rejects_bad_arguments(cuda):
    prog = api.IcProgram(SOD)
    eng = api.Engine(1, "fvchar", capacity_blocks=8, max_cases=1)
    with pytest.raises(N.AlpacaError):
        eng.add_case_expr(prog, (0,), 0.1, N.Material.make(1.4))
    with pytest.raises(N.AlpacaError):
        eng.add_case_expr(prog, (4,), 0.1, N.Material.make(1.4), units=N.Units(0.0, 1.0, 1.0))
    eng.close()
    prog.close()
