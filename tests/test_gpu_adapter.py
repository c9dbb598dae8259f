"""The integration guide's drop-in adapter (oracle/b200_convective_term_solver.h,
a ConvectiveTermSolver<Derived> concretization that calls alp_convective_fluxes)
compiled against the reference's own headers and run inside the reference's
object model (MaterialManager, EigenDecomposition, Block; oracle/adapter_harness.cpp),
against the reference's FiniteVolumeScheme / FluxSplittingScheme on the same
blocks (convective_term_solver.h:67-81, both called through the CRTP base with
zeroed flux arrays as SpaceSolver::UpdateFluxes does).

Linked with the fast library the flux arrays agree per field within
max|a - b| / max|b| <= 1e-12; linked with the strict build they are equal bit
for bit.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from alpaca_b200 import cases
from alpaca_b200 import native as N
from helpers import field_rel_err, filled

pytestmark = pytest.mark.gpu

FLUX_TOL = 1e-12


def adapter(variant, strict):
    path = os.path.join(oracle.REF_DIR,
                        f"libalpadapter_{'strict_' if strict else ''}d3_{variant}.so")
    if not os.path.exists(path) or not oracle.Reference.available(3, variant):
        pytest.skip("adapter / reference libraries not built (reference sources absent)")
    lib = C.CDLL(path)
    lib.adapter_fluxes.restype = C.c_int
    lib.adapter_fluxes.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int,
                                   C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    lib.adapter_last_error.restype = C.c_char_p
    return lib


def adapter_fluxes(lib, u, gamma, B, safe, h, precision=N.FP64):
    nb = u.shape[0]
    shape = (nb, 5, 17, 17, 17)
    fx, fy, fz = (np.full(shape, np.nan) for _ in range(3))
    rc = lib.adapter_fluxes(u.ctypes.data, nb, gamma, B, int(safe), h, fx.ctypes.data,
                            fy.ctypes.data, fz.ctypes.data, precision)
    assert rc == 0, lib.adapter_last_error().decode()
    return fx, fy, fz


CASES = {
    "gas": lambda: (cases.fourier_shock(2, dim=3, seed=21), False),
    "water_safe": lambda: (cases.water_spheres(2, seed=22), True),
}


@pytest.mark.parametrize("variant", ["fvchar", "fvprim", "fsroe"])
@pytest.mark.parametrize("which", list(CASES))
@pytest.mark.parametrize("strict", [False, True])
def test_adapter_fluxes_equal_reference_scheme(cuda, variant, which, strict):
    lib = adapter(variant, strict)
    case, safe = CASES[which]()
    u = np.ascontiguousarray(filled(case))
    h = case.grid.cell_size
    ref = oracle.Reference(3, variant).space_rhs(u, case.gamma, case.B, safe, h)[:3]
    got = adapter_fluxes(lib, u, case.gamma, case.B, safe, h)
    for a, b in zip(got, ref):
        if strict:
            assert np.array_equal(a, b)
        else:
            err = field_rel_err(a, b)
            assert err.max() <= FLUX_TOL, err


def test_adapter_reports_library_errors(cuda):
    """A selection the library refuses (an invalid material here) comes back
    as the adapter's exception, with the library's message."""
    lib = adapter("fvchar", False)
    case = cases.fourier_shock(1, dim=3, seed=23)
    u = np.ascontiguousarray(filled(case))
    nb = u.shape[0]
    f = [np.zeros((nb, 5, 17, 17, 17)) for _ in range(3)]
    rc = lib.adapter_fluxes(u.ctypes.data, nb, 1.4, 0.0, 0, case.grid.cell_size, f[0].ctypes.data,
                            f[1].ctypes.data, f[2].ctypes.data, 7)
    assert rc == -1
    assert "precision" in lib.adapter_last_error().decode().lower()
