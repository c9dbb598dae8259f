"""Checkpoint and resume of engine cases (alp_engine_checkpoint_case /
alp_engine_restore_case): a case written to a checkpoint file after some
steps and restored into a new engine ends exactly where the uninterrupted case
ends, bit for bit, with the same time and step count."""
import numpy as np
import pytest

from alpaca_b200 import api, cases
from alpaca_b200 import native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_resumed_case_equals_uninterrupted(cuda, tmp_path, dim):
    case = {1: cases.sod_1d(), 2: cases.fourier_shock(2, dim=2, seed=3),
            3: cases.fourier_shock(1, dim=3, seed=5)}[dim]
    I = cases.interior(dim)
    # uninterrupted: 20 steps, then the step budget of 25 ends the case
    a = api.Engine(dim, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    ca = a.add_case(case, max_steps=25)
    a.step(20)
    mid_ref = a.get(ca)
    a.step(10)
    ua, ta, sa = a.get(ca)
    a.close()
    # interrupted after 20 steps, written to a file, resumed in a new engine
    b = api.Engine(dim, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    cb = b.add_case(case, max_steps=25)
    b.step(20)
    path = str(tmp_path / "ck.npz")
    api.save_checkpoint(path, b.checkpoint(cb))
    b.close()
    ck = api.load_checkpoint(path)
    assert ck["steps"] == 20 and ck["t"] == mid_ref[1]
    assert np.array_equal(ck["blocks"][I], mid_ref[0][I])
    c = api.Engine(dim, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    cc = c.restore(ck)
    c.step(10)
    uc, tc, sc = c.get(cc)
    c.close()
    assert sa == sc == 25 and ta == tc
    assert np.array_equal(ua[I], uc[I])


def test_restore_rejects_another_dimension(cuda):
    case = cases.sod_1d()
    e = api.Engine(1, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    ck = e.checkpoint(e.add_case(case))
    e.close()
    e2 = api.Engine(2, "fvchar", capacity_blocks=64, max_cases=1)
    with pytest.raises(N.AlpacaError):
        e2.restore(ck)
    e2.close()


@pytest.mark.parametrize("other", [("fsroe", N.FP64, None), ("fvchar", N.FP32_FLUX, None),
                                   ("fvchar", N.FP64, N.RK2)])
def test_restore_rejects_another_scheme(cuda, other):
    """A case checkpointed under FV char / FP64 / RK3 is refused by an engine
    with another scheme, precision or time integrator, and accepted by one
    with the same selection."""
    case = cases.fourier_shock(1, dim=3, seed=6)
    e = api.Engine(3, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    ck = e.checkpoint(e.add_case(case))
    e.close()
    variant, precision, integrator = other
    sch = N.Scheme.make(variant, precision)
    if integrator is not None:
        sch.time_integrator = integrator
    e2 = api.Engine(3, sch, precision=precision, capacity_blocks=case.grid.nb, max_cases=1)
    with pytest.raises(N.AlpacaError, match="scheme selection"):
        e2.restore(ck)
    e2.close()
    e3 = api.Engine(3, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    e3.restore(ck)
    e3.close()


def test_resumed_level_case_equals_uninterrupted(cuda):
    """A three-level 2D tree checkpointed after one macro step and resumed in a
    new level engine ends where three uninterrupted macro steps end."""
    c = cases.spherical_shock_levels(n0=4, dim=2, lmax=2)
    a = api.LevelEngine(c, "fvchar", max_macro=3)
    a.step(3)
    ua, ta, ma = a.get()
    a.close()
    b = api.LevelEngine(c, "fvchar", max_macro=3)
    b.step(1)
    ck = b.checkpoint()
    r = b.restore(ck)
    b.close()
    r.step(5)  # two macro steps are left
    ur, tr, mr = r.get()
    r.close()
    I = cases.interior(2)
    assert ma == 3 and ck["macro"] == 1 and mr == 2
    assert ta == tr
    assert np.array_equal(ua[I], ur[I])


def test_restore_beside_a_running_case(cuda):
    """Restored into an engine that already runs another case (so at another
    place in the block pool): the restored case still ends where the
    uninterrupted one ends, and the other case is untouched."""
    sod = cases.sod_1d()
    other = cases.sod_1d(nblocks=6)
    ref = api.Engine(1, "fvchar", capacity_blocks=16, max_cases=2)
    r = ref.add_case(sod)
    ref.step(30)
    u_ref, t_ref, s_ref = ref.get(r)
    ref.close()
    a = api.Engine(1, "fvchar", capacity_blocks=16, max_cases=2)
    ca = a.add_case(sod)
    a.step(12)
    ck = a.checkpoint(ca)
    a.close()
    b = api.Engine(1, "fvchar", capacity_blocks=32, max_cases=3)
    ob = b.add_case(other)
    b.step(5)
    cb = b.restore(ck)
    b.step(18)
    u, t, s = b.get(cb)
    uo, to, so = b.get(ob)
    b.close()
    solo = api.Engine(1, "fvchar", capacity_blocks=16, max_cases=1)
    oo = solo.add_case(other)
    solo.step(23)
    u_solo, t_solo, s_solo = solo.get(oo)
    solo.close()
    I = cases.interior(1)
    assert s == s_ref == 30 and t == t_ref and np.array_equal(u[I], u_ref[I])
    assert so == s_solo == 23 and to == t_solo and np.array_equal(uo[I], u_solo[I])
