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
    # 1st call: the largest 3D batch that fits (27 blocks), 2nd call: a
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
