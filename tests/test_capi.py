"""The C-ABI library without a GPU: it loads, exports every function the
header declares, and rejects bad arguments before touching the device."""
import ctypes as C

import pytest

from alpaca_b200 import native as N


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    declared = N.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_default_scheme():
    assert b"sm_100a" in N.lib().alp_version()
    s = N.Scheme()
    N.lib().alp_scheme_default(C.byref(s))
    assert (s.convective_term_solver, s.state_reconstruction, s.reconstruction_stencil,
            s.riemann_solver, s.signal_speed, s.flux_splitting, s.time_integrator,
            s.precision) == (N.FINITE_VOLUME, N.RECON_CHARACTERISTIC, N.STENCIL_WENO5,
                             N.RIEMANN_HLLC, N.SIGNAL_SPEED_EINFELDT, N.FLUX_SPLITTING_ROE,
                             N.RK3, N.FP64)


def test_invalid_arguments_are_rejected_without_gpu():
    lib = N.lib()
    mat = N.Material.make(1.4)
    sch = N.Scheme.make("fvchar")
    null = C.c_void_p(0)
    rc = lib.alp_convective_fluxes(4, C.byref(sch), C.byref(mat), null, 1, 0.1, null, null, null, null)
    assert rc == N.ALP_ERR_INVALID and b"dim" in lib.alp_last_error()
    bad = N.Scheme.make("fvchar")
    bad.reconstruction_stencil = 14  # WENO9 is not compiled
    rc = lib.alp_convective_fluxes(3, C.byref(bad), C.byref(mat), null, 1, 0.1, null, null, null, null)
    assert rc == N.ALP_ERR_INVALID and b"WENO5" in lib.alp_last_error()
    cons = N.Scheme.make("fvchar")
    cons.state_reconstruction = N.RECON_CONSERVATIVE
    rc = lib.alp_convective_fluxes(3, C.byref(cons), C.byref(mat), null, 1, 0.1, null, null, null, null)
    assert rc == N.ALP_ERR_INVALID
    badmat = N.Material.make(1.0)
    rc = lib.alp_convective_fluxes(3, C.byref(sch), C.byref(badmat), null, 1, 0.1, null, null, null, null)
    assert rc == N.ALP_ERR_INVALID and b"gamma" in lib.alp_last_error()
    rc = lib.alp_rk3_stage(3, null, null, null, 1, 3, 0.1, null)
    assert rc == N.ALP_ERR_INVALID
    rc = lib.alp_halo_update(3, null, 1, 5, null, 7, null)
    assert rc == N.ALP_ERR_INVALID
    h = C.c_void_p()
    assert lib.alp_engine_create(3, C.byref(sch), 0, 1, C.byref(h)) == N.ALP_ERR_INVALID


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_workspace_and_engine_sizes(dim):
    lib = N.lib()
    faces = 17 * (17 if dim > 1 else 2) * (17 if dim > 2 else 2)
    assert lib.alp_space_rhs_workspace_size(dim, 7) == 7 * dim * (dim + 2) * faces * 8
    cells = 24 ** dim
    per_block = 3 * (dim + 2) * cells * 8 + (dim + 2) * 16 ** dim * 8
    assert lib.alp_engine_bytes(dim, 10, 2) >= 10 * per_block


def test_struct_layouts_match_the_header(tmp_path):
    """ctypes mirrors of the ABI structs have the C sizes and field offsets."""
    import os
    import subprocess
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "alpaca_b200.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(alp_scheme),'
        ' sizeof(alp_material), sizeof(alp_request), sizeof(alp_result), sizeof(alp_server_config),'
        ' offsetof(alp_request, ic_params), offsetof(alp_request, arrival_s),'
        ' offsetof(alp_server_config, scheme)); return 0;}\n')
    inc = os.path.join(os.path.dirname(N.HEADER))
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", inc, str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    want = [C.sizeof(N.Scheme), C.sizeof(N.Material), C.sizeof(N.Request), C.sizeof(N.Result),
            C.sizeof(N.ServerConfig), N.Request.ic_params.offset, N.Request.arrival_s.offset,
            N.ServerConfig.scheme.offset]
    assert got == want


def test_serve_rejects_bad_config_without_gpu():
    cfg = N.ServerConfig()
    cfg.steps_per_poll = 0
    cfg.max_cases = 4
    rc = N.lib().alp_serve(C.byref(cfg), None, 0, None, None)
    assert rc == N.ALP_ERR_INVALID
    cfg.steps_per_poll = 4
    cfg.shortest_first = 1
    cfg.step_set_cells = 0.0
    rc = N.lib().alp_serve(C.byref(cfg), None, 0, None, None)
    assert rc == N.ALP_ERR_INVALID and b"step_set_cells" in N.lib().alp_last_error()


def test_request_stream_is_seeded_and_in_range():
    from alpaca_b200 import serving
    a = serving.request_stream(40, seed=3)
    b = serving.request_stream(40, seed=3)
    assert [(r.kind, r.nblocks, r.max_steps) for r in a] == [(r.kind, r.nblocks, r.max_steps) for r in b]
    assert all(1 <= r.blocks <= 2600 and 200 <= r.max_steps <= 2000 for r in a)
    assert all(a[i].arrival_s < a[i + 1].arrival_s for i in range(39))
    water = [r for r in a if r.kind == "blast3d_water"]
    assert water and abs(water[0].B - 3430.0) < 1e-9 and water[0].gamma == 6.12


def test_extension_selections_validated_on_the_host():
    """Unknown values and FP32 with a further selection are rejected before any
    device work; the further selections themselves pass validation (the call
    then only fails on the null buffers)."""
    lib = N.lib()
    mat = N.Material.make(1.4)
    ws = C.c_void_p(0)

    def rhs(sch):
        return lib.alp_space_rhs(3, C.byref(sch), C.byref(mat), None, 1, 0.1, None, ws, 0, None)

    s = N.Scheme.make("fvchar")
    s.reconstruction_stencil = 5  # WENO5AER: not compiled
    assert rhs(s) == N.ALP_ERR_INVALID and b"WENO5Z" in lib.alp_last_error()
    s = N.Scheme.make("fsroe")
    s.flux_splitting = 5  # no such splitting
    assert rhs(s) == N.ALP_ERR_INVALID and b"GlobalLaxFriedrichs" in lib.alp_last_error()
    s = N.Scheme.make("fvchar_teno5", N.FP32_FLUX)
    assert rhs(s) == N.ALP_ERR_INVALID and b"FP32_FLUX" in lib.alp_last_error()
    for name in N.EXT_SCHEMES:
        assert rhs(N.Scheme.make(name)) == N.ALP_ERR_INVALID
        assert b"null buffer" in lib.alp_last_error(), name
