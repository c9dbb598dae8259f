"""Fifth-order prediction of child cells from parent cells
(Multiresolution::Prediction, multiresolution.cpp:146-283): the oracle's
restatement against the reference's own function, bit for bit, and two
properties of the scheme (exact for cell averages of polynomials of degree 4,
and conservative: the children's mean is the parent cell).
"""
import numpy as np
import pytest

import oracle

TC = 24
# child cell ranges as the reference's halo managers pass them (start, count):
# face halos West / East, a South face, the interior, a corner
REGIONS = [((0, 4, 4), (4, 16, 16)), ((20, 4, 4), (4, 16, 16)), ((4, 0, 4), (16, 4, 16)),
           ((4, 4, 4), (16, 16, 16)), ((0, 0, 0), (4, 4, 4)), ((4, 20, 20), (16, 4, 4))]


def shape(dim):
    return (TC,) * dim + (1,) * (3 - dim)


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_restatement_is_the_reference(dim):
    if not oracle.Reference.available(dim):
        pytest.skip("reference library not built")
    rng = np.random.default_rng(dim)
    ref, res = oracle.Reference(dim), oracle.Restatement(dim)
    for _ in range(2):
        parent = rng.standard_normal(shape(dim)) * rng.uniform(0.1, 10.0)
        for octant in range(1 << dim):
            for st, ct in REGIONS:
                a = ref.prediction(parent, octant, st[:dim], ct[:dim])
                b = res.prediction(parent, octant, st[:dim], ct[:dim])
                assert np.array_equal(a, b), (octant, st)
                assert np.count_nonzero(b) >= np.prod(ct[:dim]) // 2


def cell_averages(dim, n, h, x0, poly):
    """Cell averages of a tensor-product polynomial (coefficients per axis,
    highest power first) over n cells of width h from x0, per axis."""
    out = []
    for d in range(dim):
        p = np.polyint(poly[d])
        a = x0[d] + h * np.arange(n)
        out.append((np.polyval(p, a + h) - np.polyval(p, a)) / h)
    g = out[0]
    for d in range(1, dim):
        g = np.multiply.outer(g, out[d])
    return g.reshape(shape(dim)) if dim < 3 else g


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_exact_for_degree_four(dim):
    """A parent of width 2h covers children of width h: the children's
    predicted averages equal their exact averages for a quartic per axis."""
    rng = np.random.default_rng(10 + dim)
    poly = [rng.uniform(-1, 1, 5) for _ in range(dim)]
    x0 = rng.uniform(-0.5, 0.5, dim)
    H = 0.1
    parent = cell_averages(dim, TC, H, x0, poly)
    res = oracle.Restatement(dim)
    for octant in range(1 << dim):
        # the child's interior 4..19 lies over parent cells 4 + 8 * bit .. + 8,
        # so child cell c spans [x0 + H * (2 + 8 * bit) + c * H / 2, + H / 2]
        start, count = (4,) * dim, (16,) * dim
        got = res.prediction(parent, octant, start, count)
        cx0 = [x0[d] + H * (2 + 8 * ((octant >> d) & 1)) for d in range(dim)]
        exact = cell_averages(dim, TC, H / 2, cx0, poly)
        sl = tuple(slice(4, 20) for _ in range(dim))
        scale = np.abs(exact[sl]).max()
        assert np.abs(got[sl] - exact[sl]).max() <= 1e-12 * scale, octant


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_children_keep_the_parent_mean(dim):
    rng = np.random.default_rng(20 + dim)
    parent = rng.uniform(0.5, 2.0, shape(dim))
    res = oracle.Restatement(dim)
    got = res.prediction(parent, 0, (4,) * dim, (16,) * dim)
    c = got[tuple(slice(4, 20) for _ in range(dim))]
    for d in range(dim):
        c = c.reshape(c.shape[:d] + (8, 2) + c.shape[d + 1:]).mean(axis=d + 1)
    p = parent[tuple(slice(4, 12) for _ in range(dim))]
    assert np.abs(c - p).max() <= 1e-14 * np.abs(p).max()
