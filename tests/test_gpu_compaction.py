"""Engine slot compaction: when a case's blocks fit only into the free slots
taken together (the pool is fragmented by cases that left), the live cases are
moved together first. The moved case and the new one then step exactly as
each alone, bit for bit; a case larger than all free slots is still refused."""
import numpy as np
import pytest

from alpaca_b200 import api, cases
from alpaca_b200 import native as N

pytestmark = pytest.mark.gpu


def alone(case, steps):
    e = api.Engine(case.grid.dim, "fvchar", capacity_blocks=case.grid.nb, max_cases=1)
    c = e.add_case(case, max_steps=steps)
    e.step(steps)
    out = e.get(c)
    e.close()
    return out


@pytest.mark.parametrize("dim", [2, 3])
def test_fragmented_pool_is_compacted(cuda, dim):
    a = cases.fourier_shock(2, dim=dim, seed=61)  # 4 (2D) / 8 (3D) blocks
    b = cases.fourier_shock(1, dim=dim, seed=62)  # 1 block
    c = cases.fourier_shock(2, dim=dim, seed=63)
    cap = a.grid.nb + b.grid.nb + c.grid.nb
    e = api.Engine(dim, "fvchar", capacity_blocks=cap, max_cases=4)
    ia = e.add_case(a, max_steps=6)
    ib = e.add_case(b, max_steps=6)
    ic = e.add_case(c, max_steps=6)
    e.step(2)
    e.remove_case(ia)
    e.remove_case(ic)
    # free: a's slots before b and c's slots after it; a case of exactly the
    # free slots in total fits only once b has moved down
    big = cases.fourier_shock(2, dim=dim, seed=65)
    n_free = a.grid.nb + c.grid.nb
    g = cases.BlockGrid(dim, (n_free,) + (1,) * (dim - 1), (1,) * dim, 1.0 / (16 * n_free))
    x = g.cell_centres()[0]
    glob = cases.primes_to_conservatives(dim, 1.0 + 0.2 * np.sin(2 * np.pi * x), 1.0 + 0 * x,
                                         [0.3 + 0 * x] * dim, 1.4)
    wide = cases.Case("wide", g, g.scatter(glob), 1.4)
    iw = e.add_case(wide, max_steps=4)
    with pytest.raises(N.AlpacaError):   # nothing left
        e.add_case(big, max_steps=1)
    e.step(4)
    ub, tb, sb = e.get(ib)
    uw, tw, sw = e.get(iw)
    e.close()
    I = cases.interior(dim)
    rb = alone(b, 6)
    rw = alone(wide, 4)
    assert sb == 6 and sw == 4
    assert tb == rb[1] and np.array_equal(ub[I], rb[0][I])
    assert tw == rw[1] and np.array_equal(uw[I], rw[0][I])
