"""Further selections of the plugin surface on the GPU (run-time selected FP64
face kernels): reconstruction stencils WENO5-Z, TENO5, WENO3 and first order,
the HLL and HLLC-LM Riemann solvers, the Davis, Toro and arithmetic signal
speeds and the Roe-M, LLF and LLF-M flux splittings, against the oracle and
the reference's own outputs (golden fixtures).

Tolerances as for the default schemes: one RHS per field max|d| / max|ref|
<= 1e-12 (a field whose reference is identically zero, as the mass RHS of the
low-Mach splittings on a fluid at rest, against the largest field's scale);
runs per field L1 <= 1e-10. The strict build is bit-exact except
where the reference calls std::pow (Toro signal speeds) or std::sin (HLLC-LM),
whose CUDA versions may differ in the last bit: there <= 1e-13.

WENO7's smoothness indicators are quadratic forms with coefficients up to
17246 that cancel on smooth data; the fast build's fused multiply-adds round
them differently, and the nonlinear weights amplify that to a few 1e-12 of the
flux. Its fast-build RHS bound is 2e-11 (the strict build stays bit-exact).
Its epsilon is 1e-10, against a rounding residue of the indicators near 1e-12
on flat data, so over a whole Sod run those differences move the weights by up
to a percent in nearly flat regions (more under Roe-M, which does not damp a
fluid at rest): fast runs <= 1e-6 in L1, and the strict build's run is held to
the reference's final state at <= 1e-12.
"""
import os

import numpy as np
import pytest

import oracle
from alpaca_b200 import api, cases
from alpaca_b200 import native as N
from helpers import field_rel_err_floored as field_rel_err, filled, l1_rel, small_cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ext")
RHS_TOL = 1e-12
RUN_TOL = 1e-10
EXT = list(N.EXT_SCHEMES)
LIBM = {"fvchar_toro": "pow", "fvchar_hllclm": "sin"}


def rhs_tol(variant):
    return 2e-11 if "weno7" in variant else RHS_TOL


def run_tol(variant):
    return 1e-6 if "weno7" in variant else RUN_TOL


def to_dev(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("variant", EXT)
def test_ext_fluxes_and_rhs_match_oracle(cuda, dim, variant):
    case = small_cases()[dim]
    u = filled(case)
    h = case.grid.cell_size
    mat = N.Material.make(case.gamma)
    fx, fy, fz, rhs = oracle.Restatement(dim, variant).space_rhs(u, case.gamma, 0.0, False, h)
    ud = to_dev(u, cuda)
    f = api.convective_fluxes(ud, dim, variant, mat, h)
    tol = rhs_tol(variant)
    for d, ref in enumerate((fx, fy, fz)[:dim]):
        assert field_rel_err(f[d].cpu().numpy(), ref).max() <= tol, d
    r = api.space_rhs(ud, dim, variant, mat, h).cpu().numpy()
    I = cases.interior(dim)
    assert field_rel_err(r[I], rhs[I]).max() <= tol
    if dim != 2:
        z = np.load(os.path.join(GOLDEN, f"rhs_d{dim}_{variant}.npz"))
        assert field_rel_err(r[I], z["rhs"]).max() <= tol


@pytest.mark.parametrize("variant", EXT)
def test_ext_strict_build(cuda, variant):
    case = small_cases()[3]
    u = filled(case)
    h = case.grid.cell_size
    rhs = oracle.Restatement(3, variant).space_rhs(u, case.gamma, 0.0, False, h)[3]
    r = api.space_rhs(to_dev(u, cuda), 3, variant, N.Material.make(case.gamma), h,
                      strict=True).cpu().numpy()
    I = cases.interior(3)
    if variant in LIBM:
        assert field_rel_err(r[I], rhs[I]).max() <= 1e-13
    else:
        assert np.array_equal(r[I], rhs[I])


def engine_sod(variant, strict=False):
    case = cases.sod_1d()
    z = np.load(os.path.join(GOLDEN, f"sod1d_{variant}.npz"))
    eng = api.Engine(1, variant, capacity_blocks=case.grid.nb, max_cases=1, strict=strict)
    cid = eng.add_case(case)
    eng.run_to_end(chunk=50)
    got, t, steps = eng.get(cid)
    eng.close()
    assert steps == int(z["steps"]) and t == pytest.approx(float(z["t"]), rel=1e-14)
    return got[cases.interior(1)], z["final"]


@pytest.mark.parametrize("variant", EXT)
def test_ext_engine_sod_matches_reference(cuda, variant):
    """1D Sod to t = 0.2 in the engine against the reference's run."""
    g, ref = engine_sod(variant)
    for f in range(3):
        assert l1_rel(g[:, f], ref[:, f]) <= run_tol(variant), f


@pytest.mark.parametrize("variant", [v for v in EXT if "weno7" in v])
def test_weno7_strict_engine_sod_matches_reference(cuda, variant):
    """The strict build's WENO7 Sod runs against the reference's runs."""
    g, ref = engine_sod(variant, strict=True)
    for f in range(3):
        assert l1_rel(g[:, f], ref[:, f]) <= 1e-12, f


@pytest.mark.parametrize("variant", ["fvchar_teno5", "fvchar_hll", "fs_llf", "fs_roem"])
def test_ext_engine_3d(cuda, variant):
    """Five engine steps on 2x2x2 blocks against the oracle."""
    case = cases.fourier_shock(2, dim=3, seed=4)
    ref = oracle.Restatement(3, variant).run(case.u, case.grid.nbr, case.gamma, 0.0, False,
                                             case.grid.cell_size, case.cfl, 1e300, max_steps=5,
                                             nthreads=8)[0]
    eng = api.Engine(3, variant, capacity_blocks=case.grid.nb, max_cases=1)
    cid = eng.add_case(case, max_steps=5)
    eng.step(5)
    got = eng.get(cid)[0]
    eng.close()
    I = cases.interior(3)
    for f in range(5):
        assert l1_rel(got[I][:, f], ref[I][:, f]) <= RUN_TOL, f


def level_case_and_reference(variant):
    lc = cases.spherical_shock_levels(n0=4, dim=2, lmax=2)
    ref = oracle.Restatement(2, variant).levels_run(lc.u, lc.level, lc.coord, lc.n0, lc.h0,
                                                    lc.gamma, 0.0, False, lc.cfl, lc.t_end,
                                                    max_macro=1)[0]
    return lc, ref


@pytest.mark.parametrize("variant", ["fvchar_teno5", "fvchar_hll", "fs_llf"])
def test_ext_levels(cuda, variant):
    """One macro step of a three-level 2D tree against the oracle."""
    lc, ref = level_case_and_reference(variant)
    le = api.LevelEngine(lc, variant, max_macro=1)
    le.step(1)
    got = le.get()[0]
    le.close()
    I = cases.interior(2)
    for f in range(4):
        assert l1_rel(got[I][:, f], ref[I][:, f]) <= RUN_TOL, f


@pytest.mark.parametrize("variant", ["fs_roem", "fs_llfm"])
def test_low_mach_splitting_breaks_down_like_the_reference(cuda, variant):
    """Roe-M and LLF-M limit the acoustic eigenvalues to 5 |u|, so a fluid at
    rest gets no dissipation: on the spherical shock at rest the oracle's state
    goes non-finite within one macro step, and the GPU reports ALP_ERR_NUMERIC."""
    lc, ref = level_case_and_reference(variant)
    assert not np.isfinite(ref[cases.interior(2)]).all()
    le = api.LevelEngine(lc, variant, max_macro=1)
    le.step(1)
    with pytest.raises(N.AlpacaError) as err:
        le.get()
    le.close()
    assert err.value.code == N.ALP_ERR_NUMERIC
