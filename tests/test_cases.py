"""Workload generators and block-grid neighbour tables (CPU)."""
import numpy as np

from alpaca_b200 import cases


def test_periodic_neighbours_wrap():
    g = cases.BlockGrid(3, (4, 4, 4), (True, True, True), 1 / 64)
    assert (g.nbr >= 0).all() and (g.nbr26 >= 0).all()
    ids = np.arange(64).reshape(4, 4, 4)
    b = ids[0, 2, 3]
    assert g.nbr[b, 0] == ids[3, 2, 3] and g.nbr[b, 1] == ids[1, 2, 3]
    assert g.nbr[b, 5] == ids[0, 2, 0]


def test_domain_faces_are_zero_gradient():
    g = cases.BlockGrid(1, (8,), (False,), 1 / 128)
    assert g.nbr[0, 0] == -1 and g.nbr[0, 1] == 1 and g.nbr[7, 1] == -1
    assert (g.nbr[:, 2:] == -1).all()


def test_scatter_gather_round_trip():
    g = cases.BlockGrid(2, (3, 2), (True, False), 1 / 48)
    glob = np.random.default_rng(0).random((4,) + g.cells_shape())
    assert np.array_equal(g.gather(g.scatter(glob)), glob)


def test_rankine_hugoniot_mach2():
    r2, u2, p2 = cases.rankine_hugoniot(1.0, 0.0, 1.0, 1.4, 2.0)
    assert np.isclose(r2, 8 / 3) and np.isclose(p2, 4.5)
    c1 = np.sqrt(1.4)
    assert np.isclose(u2, 2 * c1 * (1 - 3 / 8))


def test_c2_case_shape_and_positivity():
    c = cases.fourier_shock(2, dim=3, seed=1)
    assert c.u.shape == (8, 5, 24, 24, 24)
    rho = c.u[cases.interior(3)][:, 0]
    assert rho.min() > 0.8
