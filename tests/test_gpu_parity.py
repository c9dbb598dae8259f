"""Parity of the CUDA path (through the C ABI) with the CPU oracle and with the
golden fixtures generated from the reference itself.

Tolerances (FP64 form):
  * one right-hand-side evaluation: per field, max|gpu - ref| / max|ref| <= 1e-12
  * after a time loop: per field, sum|gpu - ref| / sum|ref| <= 1e-10 (L1)
The only arithmetic difference from the reference is FMA contraction on the GPU.
"""
import os

import numpy as np
import pytest

import oracle
from alpaca_b200 import api, cases
from alpaca_b200 import native as N
from helpers import field_rel_err, filled, l1_rel, small_cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RHS_TOL = 1e-12
RUN_TOL = 1e-10
VARIANTS = list(oracle.VARIANTS)


def to_dev(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def l1_per_field(a, b):
    return max(l1_rel(a[:, f], b[:, f]) for f in range(a.shape[1]))


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("variant", VARIANTS)
def test_convective_fluxes_and_rhs(cuda, dim, variant):
    case = small_cases()[dim]
    u = filled(case)
    h = case.grid.cell_size
    mat = N.Material.make(case.gamma)
    fx, fy, fz, rhs = oracle.Restatement(dim, variant).space_rhs(u, case.gamma, 0.0, False, h)
    ud = to_dev(u, cuda)
    f = api.convective_fluxes(ud, dim, variant, mat, h)
    for d, ref in enumerate((fx, fy, fz)[:dim]):
        err = field_rel_err(f[d].cpu().numpy(), ref)
        assert err.max() <= RHS_TOL, (d, err)
    r = api.space_rhs(ud, dim, variant, mat, h).cpu().numpy()
    I = cases.interior(dim)
    assert field_rel_err(r[I], rhs[I]).max() <= RHS_TOL
    # halos of the RHS buffer are zero as after SpaceSolver's zeroing
    mask = np.ones(r.shape, bool)
    mask[I] = False
    assert not r[mask].any()
    # the reference's own output (golden fixture)
    z = np.load(os.path.join(GOLDEN, f"rhs_d{dim}_{variant}.npz"))
    assert field_rel_err(r[I], z["rhs"]).max() <= RHS_TOL


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("safe", [False, True])
def test_stiffened_gas_rhs(cuda, variant, safe):
    """Stiffened gas with p << gamma*B. Pressure recovery p = (gamma-1)(E - rho u^2/2)
    - gamma B cancels log10(gamma B / p) digits, so a one-ulp difference in E (FMA
    contraction on the GPU) moves p by eps * gamma * B. The FP64 tolerance is the
    1e-12 bound scaled by that condition number kappa = (p + gamma B) / p; the
    strict (no-FMA) build below matches the reference bit for bit."""
    gamma, B = 6.12, 3000.0
    case = cases.fourier_shock(1, dim=3, seed=11, gamma=gamma, B=B)
    u = filled(case)
    h = case.grid.cell_size
    rhs = oracle.Restatement(3, variant).space_rhs(u, gamma, B, safe, h)[3]
    r = api.space_rhs(to_dev(u, cuda), 3, variant, N.Material.make(gamma, B, safe), h)
    I = cases.interior(3)
    p = oracle.Restatement(3).prime_states(u, gamma, B, safe)[I][:, 1]
    kappa = float(((p + gamma * B) / np.abs(p)).max())
    assert field_rel_err(r.cpu().numpy()[I], rhs[I]).max() <= RHS_TOL * kappa


def test_accumulate_contract(cuda):
    """UpdateConvectiveFluxes adds to the caller's arrays (convective_term_solver.h:67-81)."""
    case = small_cases()[2]
    ud = to_dev(filled(case), cuda)
    mat = N.Material.make(1.4)
    f1 = api.convective_fluxes(ud, 2, "fvchar", mat, case.grid.cell_size)
    import ctypes as C
    sch = N.Scheme.make("fvchar")
    N.check(N.lib().alp_convective_fluxes(2, C.byref(sch), C.byref(mat), api._ptr(ud), case.grid.nb,
                                          case.grid.cell_size, api._ptr(f1[0]), api._ptr(f1[1]),
                                          C.c_void_p(0), api._stream()))
    f2 = api.convective_fluxes(ud, 2, "fvchar", mat, case.grid.cell_size)
    assert np.array_equal(f1[0].cpu().numpy(), 2 * f2[0].cpu().numpy())


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_prime_states(cuda, dim):
    case = small_cases()[dim]
    u = np.ascontiguousarray(case.u.copy())
    oracle.Restatement(dim).halo_fill(u, case.grid.nbr26, zero_gradient=True)  # every cell
    p = api.prime_states(to_dev(u, cuda), dim, N.Material.make(case.gamma)).cpu().numpy()
    ref = oracle.Restatement(dim).prime_states(u, case.gamma)
    assert field_rel_err(p, ref).max() <= 1e-15


def test_halo_known_answer(cuda):
    """test_internal_halo_manager.cpp:76-140 through alp_halo_update (26 regions)."""
    g = cases.BlockGrid(3, (2, 2, 2), (False, False, False), 1.0 / 32)
    u = np.zeros((g.nb, 1) + cases.block_shape(3))
    for b in range(g.nb):
        u[b] = b
    ud = to_dev(u, cuda)
    api.halo_update(ud, 3, to_dev(g.nbr26, cuda), N.HALO_ALL)
    got = ud.cpu().numpy()
    for b in range(g.nb):
        for s in range(26):
            n = g.nbr26[b, s]
            if n < 0:
                continue
            o = s if s < 13 else s + 1
            off = (o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1)
            sl = tuple(slice(20, 24) if x > 0 else slice(0, 4) if x < 0 else slice(4, 20)
                       for x in off)
            assert np.all(got[(b, 0) + sl] == n)
    # every cell, domain sides included, as the oracle's 26 regions + zero-gradient slabs
    ref = u.copy()
    oracle.Restatement(3).halo_fill(ref, g.nbr26, zero_gradient=True)
    assert np.array_equal(got, ref)


def test_symmetry_wall_halos_match_oracle(cuda):
    """Symmetry walls in x, periodic y, zero-gradient z through alp_halo_update
    (26 regions): every halo cell as the oracle's mirror (normal momentum
    negated) and zero-gradient slabs, in the reference's slab order."""
    g = cases.BlockGrid(3, (2, 2, 1), (cases.SYMMETRY, True, False), 1.0 / 32)
    rng = np.random.default_rng(11)
    u = np.ascontiguousarray(rng.standard_normal((g.nb, 5) + cases.block_shape(3)))
    ud = to_dev(u, cuda)
    api.halo_update(ud, 3, to_dev(g.nbr26, cuda), N.HALO_ALL)
    ref = u.copy()
    oracle.Restatement(3).halo_fill(ref, g.nbr26, zero_gradient=True)
    assert np.array_equal(ud.cpu().numpy(), ref)


@pytest.mark.parametrize("strict", [False, True], ids=["fast", "strict"])
def test_engine_with_symmetry_walls_matches_oracle(cuda, strict):
    """Five steps of a 3D case with symmetry walls in x and z, periodic y:
    the engine's mirrored stencil gather against the oracle's halo fill."""
    g = cases.BlockGrid(3, (2, 2, 2), (cases.SYMMETRY, True, cases.SYMMETRY), 1.0 / 32)
    rng = np.random.default_rng(12)
    x = g.cell_centres()
    shp = g.cells_shape()
    rho = 1 + 0.2 * cases.fourier_modes(rng, shp, x, 3)
    p = 1 + 0.2 * cases.fourier_modes(rng, shp, x, 3)
    vel = [0.3 * cases.fourier_modes(rng, shp, x, 3) for _ in range(3)]
    u = g.scatter(cases.primes_to_conservatives(3, rho, p, vel, 1.4))
    ref = oracle.Restatement(3, "fvchar").run(u, g.nbr, 1.4, 0.0, False, g.cell_size, 0.6,
                                             1e300, max_steps=5, nthreads=8)[0]
    eng = api.Engine(3, "fvchar", capacity_blocks=g.nb, max_cases=1, strict=strict)
    cid = eng.add_case(cases.Case("sym", g, u, 1.4, 0.0, 0.6, 1e300, 5), max_steps=5)
    eng.step(5)
    got = eng.get(cid)[0]
    eng.close()
    I = cases.interior(3)
    if strict:
        assert np.array_equal(got[I], ref[I])
    else:
        for f in range(5):
            assert l1_rel(got[I][:, f], ref[I][:, f]) <= 1e-10, f


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_face_halo_update_matches_oracle(cuda, dim):
    case = small_cases()[dim]
    u = np.ascontiguousarray(case.u.copy())
    ud = to_dev(u, cuda)
    api.halo_update(ud, dim, to_dev(case.grid.nbr26, cuda), N.HALO_FACES)
    ref = u.copy()
    oracle.Restatement(dim).halo_update(ref, case.grid.nbr)
    got = ud.cpu().numpy()
    # compare interiors and the face slabs over the interior extent
    for f in range(2 * dim):
        d, hi = f // 2, f % 2
        sl = [slice(4, 20) if x < dim else slice(0, 1) for x in range(3)]
        sl[d] = slice(20, 24) if hi else slice(0, 4)
        idx = (slice(None), slice(None)) + tuple(sl)
        assert np.array_equal(got[idx], ref[idx]), f


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_timestep_size(cuda, dim):
    case = small_cases()[dim]
    u = filled(case)
    mat = N.Material.make(case.gamma)
    dt = api.timestep_size(to_dev(u, cuda), dim, mat, case.grid.cell_size, 0.6)
    ref = oracle.Restatement(dim).timestep(u, case.gamma, 0.0, False, case.grid.cell_size, 0.6)
    assert abs(dt - ref) <= 1e-15 * ref
    # end-time clip (modular_algorithm_assembler.cpp:1971-1982)
    dt2 = api.timestep_size(to_dev(u, cuda), dim, mat, case.grid.cell_size, 0.6, t=1.0,
                            t_end=1.0 + ref / 3)
    assert abs(dt2 - ref / 3) <= 1e-15


def test_rk3_stage_from_rhs(cuda):
    """TimeIntegrator stage on an oracle RHS buffer."""
    import torch
    case = small_cases()[3]
    u = filled(case)
    rhs = oracle.Restatement(3).space_rhs(u, 1.4, 0.0, False, case.grid.cell_size)[3]
    ud, u0 = to_dev(u, cuda), torch.zeros(u.shape, dtype=torch.float64, device=cuda)
    rd = to_dev(rhs, cuda)
    api.rk3_stage(ud, u0, rd, 3, 0, 1e-3)
    I = cases.interior(3)
    exp = u + 1e-3 * rhs
    assert np.allclose(ud.cpu().numpy()[I], exp[I], rtol=1e-15, atol=1e-15)
    assert np.array_equal(u0.cpu().numpy()[I], u[I])
    api.rk3_stage(ud, u0, rd, 3, 1, 1e-3)
    exp2 = 0.25 * exp + 0.75 * u + 0.25 * 1e-3 * rhs
    assert np.allclose(ud.cpu().numpy()[I], exp2[I], rtol=1e-15, atol=1e-15)


@pytest.mark.parametrize("variant", VARIANTS)
def test_engine_sod_to_end_time(cuda, variant):
    """Config 1: 1D Sod, 8 x 16 cells, WENO5 + SSP-RK3, CFL 0.6, t_end 0.2."""
    z = np.load(os.path.join(GOLDEN, f"sod1d_{variant}.npz"))
    case = cases.sod_1d()
    eng = api.Engine(1, variant, capacity_blocks=16, max_cases=2)
    cid = eng.add_case(case)
    eng.run_to_end(chunk=8)
    u, t, steps = eng.get(cid)
    eng.close()
    assert steps == int(z["steps"])
    assert abs(t - float(z["t"])) <= 1e-15
    I = cases.interior(1)
    assert l1_per_field(u[I], z["final"]) <= RUN_TOL


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("variant", VARIANTS)
def test_engine_short_run_vs_reference(cuda, dim, variant):
    z = np.load(os.path.join(GOLDEN, f"run5_d{dim}_{variant}.npz"))
    case = small_cases()[dim]
    eng = api.Engine(dim, variant, capacity_blocks=8, max_cases=2)
    cid = eng.add_case(case, max_steps=5)
    eng.run_to_end(chunk=5)
    u, t, steps = eng.get(cid)
    eng.close()
    assert steps == 5 and abs(t - float(z["t"])) <= 1e-13 * t
    I = cases.interior(dim)
    assert field_rel_err(u[I], z["final"]).max() <= RHS_TOL * 10
    assert l1_per_field(u[I], z["final"]) <= RUN_TOL


@pytest.mark.parametrize("variant", ["fvchar", "fsroe"])
def test_engine_100_steps_vs_oracle(cuda, variant):
    """100 SSP-RK3 steps of a 2x2x2-block periodic Fourier + Mach-2 case."""
    case = cases.fourier_shock(2, dim=3, seed=7)
    ref, t_ref, n_ref, _ = oracle.Restatement(3, variant).run(
        case.u, case.grid.nbr, case.gamma, 0.0, False, case.grid.cell_size, case.cfl, 1e300,
        max_steps=100, nthreads=os.cpu_count() or 1)
    eng = api.Engine(3, variant, capacity_blocks=8, max_cases=1)
    cid = eng.add_case(case, max_steps=100)
    eng.run_to_end(chunk=25)
    u, t, steps = eng.get(cid)
    eng.close()
    assert steps == n_ref == 100
    assert abs(t - t_ref) <= 1e-12 * t_ref
    I = cases.interior(3)
    assert l1_per_field(u[I], ref[I]) <= RUN_TOL


def test_engine_mix_equals_alone(cuda):
    """Cases sharing an engine give the same bits as each case alone."""
    a = cases.fourier_shock(2, dim=3, seed=21, steps=7)
    b = cases.fourier_shock(1, dim=3, seed=22, steps=4)
    out = {}
    for name, group in (("alone_a", [a]), ("alone_b", [b]), ("mix", [a, b])):
        eng = api.Engine(3, "fvchar", capacity_blocks=16, max_cases=4)
        ids = [eng.add_case(c) for c in group]
        eng.run_to_end(chunk=4)
        out[name] = [eng.get(i) for i in ids]
        eng.close()
    assert np.array_equal(out["mix"][0][0], out["alone_a"][0][0])
    assert np.array_equal(out["mix"][1][0], out["alone_b"][0][0])
    assert out["mix"][0][2] == 7 and out["mix"][1][2] == 4


def test_engine_graph_equals_eager(cuda):
    c = cases.fourier_shock(1, dim=3, seed=5, steps=3)
    res = []
    for graph in (True, False):
        eng = api.Engine(3, "fvprim", capacity_blocks=2, max_cases=1, graph=graph)
        cid = eng.add_case(c)
        eng.run_to_end(chunk=3)
        res.append(eng.get(cid)[0])
        eng.close()
    assert np.array_equal(res[0], res[1])


def test_engine_numeric_fault_is_reported(cuda):
    """A negative density stops the case and is reported through the status
    word (ALP_ERR_NUMERIC), without a device fault."""
    c = cases.fourier_shock(1, dim=3, seed=5, steps=3)
    c.u[0, 0, 10, 10, 10] = -1.0
    eng = api.Engine(3, "fvchar", capacity_blocks=2, max_cases=1)
    cid = eng.add_case(c)
    eng.step(2)
    with pytest.raises(N.AlpacaError) as e:
        eng.get(cid)
    assert e.value.code == N.ALP_ERR_NUMERIC
    assert eng.all_done()
    eng.close()


def test_engine_capacity_and_removal(cuda):
    c = cases.fourier_shock(1, dim=3, seed=5, steps=1)
    eng = api.Engine(3, "fvchar", capacity_blocks=2, max_cases=4)
    i0 = eng.add_case(c)
    i1 = eng.add_case(c)
    with pytest.raises(N.AlpacaError) as e:
        eng.add_case(c)
    assert e.value.code == N.ALP_ERR_CAPACITY
    eng.remove_case(i0)
    i2 = eng.add_case(c)
    eng.run_to_end()
    assert np.array_equal(eng.get(i1)[0], eng.get(i2)[0])
    eng.close()


# ---- the strict build (no FMA contraction): bit-for-bit ----------------------

@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("variant", VARIANTS)
def test_strict_build_rhs_bit_exact(cuda, dim, variant):
    """Without FMA contraction the CUDA arithmetic reproduces the reference's
    operation order exactly: fluxes and RHS equal the reference's bits."""
    case = small_cases()[dim]
    u = filled(case)
    h = case.grid.cell_size
    mat = N.Material.make(case.gamma)
    fx, fy, fz, rhs = oracle.Restatement(dim, variant).space_rhs(u, case.gamma, 0.0, False, h)
    ud = to_dev(u, cuda)
    f = api.convective_fluxes(ud, dim, variant, mat, h, strict=True)
    for d, ref in enumerate((fx, fy, fz)[:dim]):
        got = f[d].cpu().numpy()
        assert np.array_equal(got, ref), (d, np.abs(got - ref).max())
    r = api.space_rhs(ud, dim, variant, mat, h, strict=True).cpu().numpy()
    I = cases.interior(dim)
    z = np.load(os.path.join(GOLDEN, f"rhs_d{dim}_{variant}.npz"))
    assert np.array_equal(r[I], rhs[I]) and np.array_equal(r[I], z["rhs"]), \
        np.abs(r[I] - rhs[I]).max()


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("safe", [False, True])
def test_strict_build_stiffened_bit_exact(cuda, variant, safe):
    gamma, B = 6.12, 3000.0
    case = cases.fourier_shock(1, dim=3, seed=11, gamma=gamma, B=B)
    u = filled(case)
    h = case.grid.cell_size
    rhs = oracle.Restatement(3, variant).space_rhs(u, gamma, B, safe, h)[3]
    r = api.space_rhs(to_dev(u, cuda), 3, variant, N.Material.make(gamma, B, safe), h,
                      strict=True).cpu().numpy()
    I = cases.interior(3)
    assert np.array_equal(r[I], rhs[I]), np.abs(r[I] - rhs[I]).max()


@pytest.mark.parametrize("variant", VARIANTS)
def test_strict_engine_sod_bit_exact(cuda, variant):
    z = np.load(os.path.join(GOLDEN, f"sod1d_{variant}.npz"))
    case = cases.sod_1d()
    eng = api.Engine(1, variant, capacity_blocks=16, max_cases=2, strict=True)
    cid = eng.add_case(case)
    eng.run_to_end(chunk=8)
    u, t, steps = eng.get(cid)
    eng.close()
    assert steps == int(z["steps"]) and t == float(z["t"])
    assert np.array_equal(u[cases.interior(1)], z["final"])


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("variant", VARIANTS)
def test_strict_engine_short_run_bit_exact(cuda, dim, variant):
    z = np.load(os.path.join(GOLDEN, f"run5_d{dim}_{variant}.npz"))
    case = small_cases()[dim]
    eng = api.Engine(dim, variant, capacity_blocks=8, max_cases=2, strict=True)
    cid = eng.add_case(case, max_steps=5)
    eng.run_to_end(chunk=5)
    u, t, steps = eng.get(cid)
    eng.close()
    assert steps == 5 and t == float(z["t"])
    assert np.array_equal(u[cases.interior(dim)], z["final"])


# ---- the 128^3 configuration, 100 steps, against the reference's own run -----

def _c2_engine(variant, strict):
    case = cases.fourier_shock(8, dim=3, seed=1, steps=100)
    eng = api.Engine(3, variant, capacity_blocks=512, max_cases=1, strict=strict)
    cid = eng.add_case(case)
    eng.run_to_end(chunk=50)
    u, t, steps = eng.get(cid)
    eng.close()
    return case, u, t, steps


@pytest.mark.parametrize("variant", ["fvchar", "fsroe"])
def test_engine_c2_128cubed_100_steps(cuda, variant):
    """Config 2 at full size: 512 blocks, 100 SSP-RK3 steps, compared with the
    reference's run (per-block interior sums and every 8th cell, committed by
    tests/golden/make_golden.py --c2): L1 <= 1e-10 per field."""
    z = np.load(os.path.join(GOLDEN, f"c2_128_{variant}_100steps.npz"))
    case, u, t, steps = _c2_engine(variant, False)
    assert steps == 100 and abs(t - float(z["t"])) <= 1e-12 * t
    glob = case.grid.gather(u)
    sub = glob[:, ::8, ::8, ::8]
    for f in range(5):
        assert l1_rel(sub[f], z["sub"][f]) <= RUN_TOL, f
    sums = u[cases.interior(3)].sum(axis=(2, 3, 4))
    for f in range(5):
        assert l1_rel(sums[:, f], z["block_sums"][:, f]) <= RUN_TOL, f


def test_strict_engine_c2_bit_exact(cuda):
    z = np.load(os.path.join(GOLDEN, "c2_128_fvchar_100steps.npz"))
    case, u, t, steps = _c2_engine("fvchar", True)
    assert steps == 100 and t == float(z["t"])
    glob = case.grid.gather(u)
    assert np.array_equal(glob[:, ::8, ::8, ::8], z["sub"])
    assert np.array_equal(u[cases.interior(3)].sum(axis=(2, 3, 4)), z["block_sums"])


# ---- FP32-flux form ---------------------------------------------------------

@pytest.mark.parametrize("variant", VARIANTS)
def test_fp32_flux_rhs(cuda, variant):
    """Reconstruction and Riemann arithmetic in FP32 (increments against the
    face's left cell), state and pressure recovery in FP64: one RHS within
    1e-5 of the FP64 oracle, per field, normwise."""
    case = small_cases()[3]
    u = filled(case)
    h = case.grid.cell_size
    rhs = oracle.Restatement(3, variant).space_rhs(u, case.gamma, 0.0, False, h)[3]
    r = api.space_rhs(to_dev(u, cuda), 3, variant, N.Material.make(case.gamma), h,
                      precision=N.FP32_FLUX).cpu().numpy()
    I = cases.interior(3)
    err = field_rel_err(r[I], rhs[I])
    print(variant, "fp32 rhs rel err per field", err)
    assert err.max() <= 1e-5


@pytest.mark.parametrize("variant", VARIANTS)
def test_fp32_flux_rhs_water(cuda, variant):
    """Stiffened-gas water spheres (pressure up to 1e9 Pa against a 1e5 Pa
    background, B = 3.43e8 Pa): the FP32-flux RHS against the FP64 oracle,
    per field, normwise. The increments of a face reach ~1e4 of the
    background pressure scale, where the float WENO5 weights take their
    exponent rescaling."""
    case = cases.water_spheres(2, seed=9, p_max=1e9)
    u = filled(case)
    h = case.grid.cell_size
    rhs = oracle.Restatement(3, variant).space_rhs(u, case.gamma, case.B, True, h)[3]
    r = api.space_rhs(to_dev(u, cuda), 3, variant, N.Material.make(case.gamma, case.B, safe=True),
                      h, precision=N.FP32_FLUX).cpu().numpy()
    I = cases.interior(3)
    err = field_rel_err(r[I], rhs[I])
    print(variant, "fp32 water rhs rel err per field", err)
    assert err.max() <= 1e-5


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("precision", [N.FP64, N.FP32_FLUX])
@pytest.mark.parametrize("fluid", ["gas", "water"])
def test_free_stream_rhs_is_zero(cuda, variant, precision, fluid):
    """A uniform moving state is kept exactly: every face sees the same
    stencil, so all fluxes of a direction are equal and the divergence is 0 in
    both precisions, whatever the rounding inside the face arithmetic
    (characteristic projection, the packed FP32 WENO5 and back-projection,
    HLLC or flux splitting; ideal gas and stiffened-gas water)."""
    gamma, B = (1.4, 0.0) if fluid == "gas" else (6.12, 3.43e3)
    rho, p, vel = (1.3, 2.5, (0.4, -0.7, 0.25)) if fluid == "gas" else (1.0, 1.2e2, (3.0, 1.0, -2.0))
    e = (p + gamma * B) / (gamma - 1.0) + 0.5 * rho * sum(v * v for v in vel)
    u = np.empty((3, 5) + cases.block_shape(3))
    u[:, 0], u[:, 1] = rho, e
    for d in range(3):
        u[:, 2 + d] = rho * vel[d]
    r = api.space_rhs(to_dev(u, cuda), 3, variant, N.Material.make(gamma, B), 1.0 / 64,
                      precision=precision).cpu().numpy()
    assert np.array_equal(r[cases.interior(3)], np.zeros_like(r[cases.interior(3)]))


@pytest.mark.parametrize("variant", VARIANTS)
def test_fp32_flux_sod_density_l1(cuda, variant):
    """The precision target: relative L1 density error <= 1e-5 against the
    FP64 reference after a full run (1D Sod to t = 0.2)."""
    z = np.load(os.path.join(GOLDEN, f"sod1d_{variant}.npz"))
    eng = api.Engine(1, variant, precision=N.FP32_FLUX, capacity_blocks=16, max_cases=1)
    cid = eng.add_case(cases.sod_1d())
    eng.run_to_end(chunk=16)
    u, t, steps = eng.get(cid)
    eng.close()
    rho = u[cases.interior(1)][:, 0]
    err = l1_rel(rho, z["final"][:, 0])
    print(variant, "fp32 sod density L1", err, "steps", steps, int(z["steps"]))
    assert abs(t - 0.2) <= 1e-15 and err <= 1e-5


@pytest.mark.parametrize("variant", ["fvchar", "fsroe"])
def test_fp32_flux_3d_100_steps(cuda, variant):
    z = np.load(os.path.join(GOLDEN, f"c2_128_{variant}_100steps.npz"))
    case = cases.fourier_shock(8, dim=3, seed=1, steps=100)
    eng = api.Engine(3, variant, precision=N.FP32_FLUX, capacity_blocks=512, max_cases=1)
    cid = eng.add_case(case)
    eng.run_to_end(chunk=50)
    u, t, steps = eng.get(cid)
    eng.close()
    sub = case.grid.gather(u)[:, ::8, ::8, ::8]
    errs = [l1_rel(sub[f], z["sub"][f]) for f in range(5)]
    print(variant, "fp32 128^3 100-step L1 per field", errs)
    assert steps == 100 and errs[0] <= 1e-5


# ---- stepping candidates and the autotuner -----------------------------------

def test_autotune_leaves_state_and_candidates_agree(cuda):
    """Autotuning runs uncommitted trial steps (state and time unchanged); every
    candidate advances the case to the same result within the FP64 tolerance
    (face paths, one launch or overlapped batches, and the fused tile stages
    with 16 or 12 warps, bit-identical to each other; the pencil path sums the
    three flux differences in a different order)."""
    case = cases.fourier_shock(2, dim=3, seed=31, steps=6)
    eng = api.Engine(3, "fvchar", capacity_blocks=8, max_cases=1)
    cid = eng.add_case(case)
    eng.step(2)
    before = eng.get(cid)
    chosen, ms = eng.autotune(trial_steps=2)
    after = eng.get(cid)
    assert chosen in range(N.STEP_CANDIDATES) and all(m > 0 for m in ms)
    assert eng.path == chosen
    assert np.array_equal(before[0], after[0]) and before[1:] == after[1:]
    results = []
    for cand in range(N.STEP_CANDIDATES):
        e = api.Engine(3, "fvchar", capacity_blocks=8, max_cases=1)
        i = e.add_case(case)
        e.set_path(cand)
        e.run_to_end(chunk=6)
        results.append(e.get(i))
        e.close()
    eng.close()
    I = cases.interior(3)
    for cand in (1, 3, 4, 5):
        assert np.array_equal(results[0][0][I], results[cand][0][I]), cand
        assert results[0][1:] == results[cand][1:], cand
    assert l1_per_field(results[2][0][I], results[0][0][I]) <= 1e-13


@pytest.mark.parametrize("variant", ["fvchar", "fsroe"])
def test_overlapped_batches_strict_bit_exact(cuda, variant):
    """Face fluxes and stage updates overlapped in batches (strict build)
    reproduce the oracle bit for bit over 6 steps of a 6x6x6-block 3D case
    (216 blocks: three batches)."""
    case = cases.fourier_shock(6, dim=3, seed=32, steps=6)
    ref = oracle.Restatement(3, variant).run(case.u, case.grid.nbr, case.gamma, 0.0, False,
                                             case.grid.cell_size, case.cfl, 1e300, max_steps=6,
                                             nthreads=os.cpu_count() or 8)
    e = api.Engine(3, variant, capacity_blocks=case.grid.nb, max_cases=1, strict=True)
    i = e.add_case(case)
    e.set_path(3)
    e.run_to_end(chunk=6)
    got, t, steps = e.get(i)
    e.close()
    I = cases.interior(3)
    assert steps == 6 and t == ref[1]
    assert np.array_equal(got[I], ref[0][I])
