"""alp_space_rhs_static (face-flux scratch in a fixed device array of the
library, no allocation) against alp_space_rhs with a caller workspace, both
through the C ABI. Collected last so it also runs after every other GPU test
has used the library; it passes alone in a fresh process as well.

Tolerance as for one right-hand-side evaluation elsewhere in the suite:
per field max|a - b| / max|b| <= 1e-12 (the two calls run the same kernels).
"""
import ctypes as C

import numpy as np
import pytest

from alpaca_b200 import cases
from alpaca_b200 import native as N
from helpers import field_rel_err, filled

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
MAX_BLOCKS = {1: 10280, 2: 453, 3: 28}  # 16 MiB of [nb][dim][NE][faces] doubles


def _dev(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def rhs_workspace(dim, variant, mat, ud, h):
    import torch
    lib = N.lib()
    nb = ud.shape[0]
    ws = torch.empty(lib.alp_space_rhs_workspace_size(dim, nb) // 8, dtype=torch.float64,
                     device=ud.device)
    rhs = torch.full_like(ud, np.nan)
    sch = N.Scheme.make(variant)
    N.check(lib.alp_space_rhs(dim, C.byref(sch), C.byref(mat), ud.data_ptr(), nb, h,
                              rhs.data_ptr(), ws.data_ptr(), ws.numel() * 8, None))
    torch.cuda.synchronize()
    return rhs.cpu().numpy()


def rhs_static(dim, variant, mat, ud, h):
    import torch
    lib = N.lib()
    rhs = torch.full_like(ud, np.nan)
    sch = N.Scheme.make(variant)
    N.check(lib.alp_space_rhs_static(dim, C.byref(sch), C.byref(mat), ud.data_ptr(),
                                     ud.shape[0], h, rhs.data_ptr(), None))
    torch.cuda.synchronize()
    return rhs.cpu().numpy()


def assert_same_rhs(dim, a, b):
    I = cases.interior(dim)
    err = field_rel_err(a[I], b[I])
    assert err.max() <= RHS_TOL, err
    mask = np.ones(a.shape, bool)
    mask[I] = False
    assert not a[mask].any()  # halos zeroed as by alp_space_rhs


def test_static_scratch_matches_workspace_on_consecutive_calls(cuda):
    # 1st call: a 27-block 3D batch, 2nd call: a
    # different single block, so the 2nd call finds the 1st call's contents in
    # the shared array; 3rd and 4th: 2D and flux splitting on other inputs.
    big = cases.fourier_shock(3, dim=3, seed=7)
    one = cases.fourier_shock(1, dim=3, seed=8)
    flat = cases.fourier_shock(2, dim=2, seed=9)
    assert big.grid.nb <= MAX_BLOCKS[3]
    calls = [(3, "fvchar", big), (3, "fvchar", one), (2, "fvprim", flat), (3, "fsroe", big)]
    for dim, variant, case in calls:
        ud = _dev(filled(case), cuda)
        mat = N.Material.make(case.gamma)
        h = case.grid.cell_size
        got = rhs_static(dim, variant, mat, ud, h)
        ref = rhs_workspace(dim, variant, mat, ud, h)
        assert_same_rhs(dim, got, ref)
    # two calls in a row on the same input give the same result
    ud = _dev(filled(one), cuda)
    mat = N.Material.make(one.gamma)
    a = rhs_static(3, "fvchar", mat, ud, one.grid.cell_size)
    b = rhs_static(3, "fvchar", mat, ud, one.grid.cell_size)
    assert_same_rhs(3, a, b)


def test_static_scratch_at_its_exact_3d_limit(cuda):
    """28 blocks in 3D (a 7 x 2 x 2 periodic grid) fill the static array."""
    g = cases.BlockGrid(3, (7, 2, 2), (1, 1, 1), 1.0 / 32)  # 3.5 x 1 x 1
    assert g.nb == MAX_BLOCKS[3]
    x, y, z = g.cell_centres()
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * x / 3.5) + 0.1 * np.cos(2 * np.pi * y)
    p = 1.0 + 0.1 * np.cos(2 * np.pi * z)
    vel = [0.3 * np.sin(2 * np.pi * y), 0.2 * np.cos(2 * np.pi * z), -0.1 + 0 * x]
    glob = cases.primes_to_conservatives(3, rho, p, vel, 1.4)
    case = cases.Case("limit28", g, g.scatter(glob), 1.4)
    ud = _dev(filled(case), cuda)
    mat = N.Material.make(1.4)
    got = rhs_static(3, "fvchar", mat, ud, g.cell_size)
    assert_same_rhs(3, got, rhs_workspace(3, "fvchar", mat, ud, g.cell_size))


def test_static_scratch_glf_and_no_allocation(cuda):
    """Global Lax-Friedrichs splitting (its stateless per-call maximum takes
    a second device slot of the library) matches alp_space_rhs; after a warm-up
    call, repeated static calls leave the device's free memory unchanged."""
    import torch
    case = cases.fourier_shock(3, dim=3, seed=11)
    ud = _dev(filled(case), cuda)
    mat = N.Material.make(case.gamma)
    h = case.grid.cell_size
    got = rhs_static(3, "fs_glf", mat, ud, h)
    assert_same_rhs(3, got, rhs_workspace(3, "fs_glf", mat, ud, h))
    lib = N.lib()
    rhs = torch.empty_like(ud)
    calls = [(v, N.Scheme.make(v)) for v in ("fvchar", "fs_glf", "fsroe")]
    for _, sch in calls:  # warm-up: every path loaded once
        N.check(lib.alp_space_rhs_static(3, C.byref(sch), C.byref(mat), ud.data_ptr(),
                                         ud.shape[0], h, rhs.data_ptr(), None))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        for _, sch in calls:
            N.check(lib.alp_space_rhs_static(3, C.byref(sch), C.byref(mat), ud.data_ptr(),
                                             ud.shape[0], h, rhs.data_ptr(), None))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_static_scratch_rejects_batches_beyond_its_size(cuda):
    lib = N.lib()
    sch = N.Scheme.make("fvchar")
    mat = N.Material.make(1.4)
    for dim, cap in MAX_BLOCKS.items():
        # rejected before any pointer is used or any kernel launched
        rc = lib.alp_space_rhs_static(dim, C.byref(sch), C.byref(mat), None, cap + 1, 0.1,
                                      None, None)
        assert rc == N.ALP_ERR_CAPACITY
        assert f"at most {cap} blocks" in lib.alp_last_error().decode()
    assert lib.alp_space_rhs_static(3, C.byref(sch), C.byref(mat), None, 0, 0.1, None,
                                    None) == N.ALP_OK
    # the argument checks of alp_space_rhs come before the capacity check
    bad = N.Material.make(-1.0)
    assert lib.alp_space_rhs_static(3, C.byref(sch), C.byref(bad), None, 1000, 0.1, None,
                                    None) == N.ALP_ERR_INVALID
    assert lib.alp_space_rhs_static(3, None, C.byref(mat), None, 1000, 0.1, None,
                                    None) == N.ALP_ERR_INVALID
