"""Interior-only case transfers (alp_engine_add_case_interior /
alp_engine_get_case_interior): a case uploaded as interiors steps exactly as
the same case uploaded as full blocks, and the interiors read back equal the
interiors of the full export, bit for bit, in 1D, 2D and 3D, also for a case
placed behind another one in the pool."""
import numpy as np
import pytest

from alpaca_b200 import api, cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_interior_transfer_equals_full_blocks(cuda, dim):
    case = {1: cases.sod_1d(), 2: cases.fourier_shock(2, dim=2, seed=31),
            3: cases.fourier_shock(2, dim=3, seed=32)}[dim]
    other = {1: cases.sod_1d(nblocks=3), 2: cases.fourier_shock(1, dim=2, seed=33),
             3: cases.fourier_shock(1, dim=3, seed=34)}[dim]
    I = cases.interior(dim)
    cap = case.grid.nb + other.grid.nb
    a = api.Engine(dim, "fvchar", capacity_blocks=cap, max_cases=2)
    ca = a.add_case(case, max_steps=7)
    a.step(7)
    ua, ta, sa = a.get(ca)
    a.close()
    b = api.Engine(dim, "fvchar", capacity_blocks=cap, max_cases=2)
    b.add_case(other, max_steps=7)  # the case under test lands behind it
    inner = np.ascontiguousarray(case.u[I])
    cb = b.add_case(case, max_steps=7, interior=inner)
    b.step(7)
    ib, tb, sb = b.get_interior(cb)
    ub, _, _ = b.get(cb)
    b.close()
    assert sa == sb == 7 and ta == tb
    assert np.array_equal(ib, ua[I])
    assert np.array_equal(ub[I], ua[I])
