"""Elastic engines and the serving loop's shared HBM budget.

An elastic engine (alp_engine_create_elastic) backs only the block slots
alp_engine_reserve asks for, in place: cases step in it exactly as in a fixed
engine, the backed memory follows the reservations, and shrinking below the
resident cases first moves them together (results unchanged) or is refused.
The serving loop sizes its 2D and 3D engines from one budget, so one
dimension may use most of it while the other is idle.
"""
import numpy as np
import pytest

from alpaca_b200 import api, cases, serving
from alpaca_b200 import native as N

pytestmark = pytest.mark.gpu
CHUNK = 32 << 20


def alone(case, steps):
    e = api.Engine(case.grid.dim, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    c = e.add_case(case, max_steps=steps)
    e.step(steps)
    out = e.get(c)
    e.close()
    return out


def test_elastic_engine_grows_and_shrinks_in_place(cuda):
    a = cases.fourier_shock(2, dim=3, seed=71)   # 8 blocks
    b = cases.fourier_shock(1, dim=3, seed=72)   # 1 block
    e = api.Engine(3, "fvchar", capacity_blocks=64, max_cases=4, elastic=True)
    assert e.capacity() == {"blocks": 0, "used": 0, "bytes": 0}
    with pytest.raises(N.AlpacaError):
        e.add_case(a, max_steps=5)
    e.reserve(9)
    c = e.capacity()
    assert c["blocks"] == 9 and c["bytes"] % CHUNK == 0 and c["bytes"] >= 9 * 5 * 24 ** 3 * 8 * 3
    ia = e.add_case(a, max_steps=5)
    ib = e.add_case(b, max_steps=5)
    e.step(2)
    with pytest.raises(N.AlpacaError):
        e.reserve(8)            # the cases hold 9 slots
    e.remove_case(ia)           # b stays at slot 8
    e.reserve(1)                # b moves to slot 0, the rest is unmapped
    assert e.capacity()["blocks"] == 1
    e.reserve(40)
    ia2 = e.add_case(a, max_steps=5)
    e.step(3)
    ub, tb, sb = e.get(ib)
    ua, ta, sa = e.get(ia2)
    e.step(2)
    ua5, _, sa5 = e.get(ia2)
    e.close()
    I = cases.interior(3)
    rb, ra3, ra5 = alone(b, 5), alone(a, 3), alone(a, 5)
    assert sb == 5 and tb == rb[1] and np.array_equal(ub[I], rb[0][I])
    assert sa == 3 and ta == ra3[1] and np.array_equal(ua[I], ra3[0][I])
    assert sa5 == 5 and np.array_equal(ua5[I], ra5[0][I])


def test_serving_shares_one_budget_between_dimensions(cuda):
    """A 2D request needing about 70 % of the budget and a 3D request needing
    about half of it: no fixed split could hold both one after the other with
    a share for each; with one shared budget both complete (the later one
    admitted once the earlier has left)."""
    rng = np.random.default_rng(5)
    per3 = N.lib().alp_engine_bytes(3, 1, 0)
    per2 = N.lib().alp_engine_bytes(2, 1, 0)
    budget = 16 * per3
    n2 = int(0.7 * budget / per2)
    side = int(np.sqrt(n2))
    q2 = serving.quadrant_request(rng, side * side, 12)
    q3 = serving.blast_request(rng, 8, 12, water=False)
    q3.arrival_s = 0.0
    q2.arrival_s = 0.0
    nb2 = q2.nblocks[0] * q2.nblocks[1]
    assert nb2 * per2 > 0.5 * budget and 8 * per3 <= 0.5 * budget + per3
    res, _, _ = api.serve([q3, q2], budget)
    assert all(r["status"] == 0 and r["steps"] == 12 for r in res), res
