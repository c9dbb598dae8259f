"""ctypes bindings of the C ABI in include/alpaca_b200.h.

The CUDA library is built in-tree (alpaca_b200/libalpaca_b200.so). Loading
fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libalpaca_b200.so")
STRICT_LIB_PATH = os.path.join(HERE, "libalpaca_b200_strict.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "alpaca_b200.h")

ALP_OK, ALP_ERR_INVALID, ALP_ERR_CUDA, ALP_ERR_CAPACITY, ALP_ERR_NOT_FOUND, ALP_ERR_NUMERIC = range(6)
ALP_ABORTED = 6
FLUX_SPLITTING, FINITE_VOLUME = 0, 1
RECON_CONSERVATIVE, RECON_PRIMITIVE, RECON_CHARACTERISTIC = 0, 1, 2
STENCIL_FIRST_ORDER, STENCIL_WENO3, STENCIL_WENO5, STENCIL_WENO5Z, STENCIL_TENO5 = 0, 1, 4, 7, 11
STENCIL_WENO7 = 13
RIEMANN_HLLC, RIEMANN_HLLC_LM, RIEMANN_HLL = 0, 1, 2
SIGNAL_SPEED_EINFELDT, SIGNAL_SPEED_DAVIS, SIGNAL_SPEED_TORO, SIGNAL_SPEED_ARITHMETIC = 0, 1, 2, 3
FLUX_SPLITTING_ROE, FLUX_SPLITTING_LLF, FLUX_SPLITTING_GLF = 0, 1, 2
FLUX_SPLITTING_ROE_M, FLUX_SPLITTING_LLF_M = 3, 4

# Further selections by name: base variant and the alp_scheme fields changed
RK2, RK3 = 0, 1  # TimeIntegrators (numerical_setup.h:26)
EXT_SCHEMES = {
    "fvchar_weno5z": ("fvchar", {"reconstruction_stencil": STENCIL_WENO5Z}),
    "fvchar_teno5": ("fvchar", {"reconstruction_stencil": STENCIL_TENO5}),
    "fvchar_weno3": ("fvchar", {"reconstruction_stencil": STENCIL_WENO3}),
    "fvchar_first": ("fvchar", {"reconstruction_stencil": STENCIL_FIRST_ORDER}),
    "fvchar_hll": ("fvchar", {"riemann_solver": RIEMANN_HLL}),
    "fvchar_hllclm": ("fvchar", {"riemann_solver": RIEMANN_HLLC_LM}),
    "fvchar_davis": ("fvchar", {"signal_speed": SIGNAL_SPEED_DAVIS}),
    "fvchar_toro": ("fvchar", {"signal_speed": SIGNAL_SPEED_TORO}),
    "fvchar_arith": ("fvchar", {"signal_speed": SIGNAL_SPEED_ARITHMETIC}),
    "fvprim_teno5": ("fvprim", {"reconstruction_stencil": STENCIL_TENO5}),
    "fs_llf": ("fsroe", {"flux_splitting": FLUX_SPLITTING_LLF}),
    "fs_roem": ("fsroe", {"flux_splitting": FLUX_SPLITTING_ROE_M}),
    "fs_llfm": ("fsroe", {"flux_splitting": FLUX_SPLITTING_LLF_M}),
    "fs_teno5": ("fsroe", {"reconstruction_stencil": STENCIL_TENO5}),
    "fvchar_weno3_hll": ("fvchar", {"reconstruction_stencil": STENCIL_WENO3,
                                    "riemann_solver": RIEMANN_HLL}),
    "fs_weno3": ("fsroe", {"reconstruction_stencil": STENCIL_WENO3}),
    "fs_llf_weno3": ("fsroe", {"reconstruction_stencil": STENCIL_WENO3,
                               "flux_splitting": FLUX_SPLITTING_LLF}),
    "fs_llfm_weno3": ("fsroe", {"reconstruction_stencil": STENCIL_WENO3,
                                "flux_splitting": FLUX_SPLITTING_LLF_M}),
    "fs_glf": ("fsroe", {"flux_splitting": FLUX_SPLITTING_GLF}),
    "fs_glf_weno5z": ("fsroe", {"reconstruction_stencil": STENCIL_WENO5Z,
                                "flux_splitting": FLUX_SPLITTING_GLF}),
    # TVD-RK2 selections of the reference's DetailedSod table
    "rk2_fvchar_weno3": ("fvchar", {"reconstruction_stencil": STENCIL_WENO3,
                                    "time_integrator": RK2}),
    "rk2_fvchar_hll_weno5z": ("fvchar", {"reconstruction_stencil": STENCIL_WENO5Z,
                                         "riemann_solver": RIEMANN_HLL, "time_integrator": RK2}),
    "rk2_fs_glf": ("fsroe", {"flux_splitting": FLUX_SPLITTING_GLF, "time_integrator": RK2}),
    "rk2_fs_llf_weno5z": ("fsroe", {"reconstruction_stencil": STENCIL_WENO5Z,
                                    "flux_splitting": FLUX_SPLITTING_LLF, "time_integrator": RK2}),
    "rk2_fs_roem_weno3": ("fsroe", {"reconstruction_stencil": STENCIL_WENO3,
                                    "flux_splitting": FLUX_SPLITTING_ROE_M,
                                    "time_integrator": RK2}),
    "rk2_fs_llfm": ("fsroe", {"flux_splitting": FLUX_SPLITTING_LLF_M, "time_integrator": RK2}),
    "rk2_fs_llfm_weno5z": ("fsroe", {"reconstruction_stencil": STENCIL_WENO5Z,
                                     "flux_splitting": FLUX_SPLITTING_LLF_M,
                                     "time_integrator": RK2}),
    # WENO7 (8-cell stencils)
    "fvchar_weno7": ("fvchar", {"reconstruction_stencil": STENCIL_WENO7}),
    "fs_roem_weno7": ("fsroe", {"reconstruction_stencil": STENCIL_WENO7,
                                "flux_splitting": FLUX_SPLITTING_ROE_M}),
    "rk2_fvchar_weno7": ("fvchar", {"reconstruction_stencil": STENCIL_WENO7,
                                    "time_integrator": RK2}),
    "rk2_fs_glf_weno7": ("fsroe", {"reconstruction_stencil": STENCIL_WENO7,
                                   "flux_splitting": FLUX_SPLITTING_GLF, "time_integrator": RK2}),
    "rk2_fs_weno7": ("fsroe", {"reconstruction_stencil": STENCIL_WENO7, "time_integrator": RK2}),
}
FP64, FP32_FLUX = 0, 1
HALO_ALL, HALO_FACES = 0, 1


class AlpacaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"alpaca_b200 error {code}: {msg}")
        self.code = code


class Scheme(C.Structure):
    """alp_scheme: the reference's user_specifications selections."""
    _fields_ = [("convective_term_solver", C.c_int), ("state_reconstruction", C.c_int),
                ("reconstruction_stencil", C.c_int), ("riemann_solver", C.c_int),
                ("signal_speed", C.c_int), ("flux_splitting", C.c_int),
                ("time_integrator", C.c_int), ("precision", C.c_int)]

    @classmethod
    def make(cls, variant: str = "fvchar", precision: int = FP64) -> "Scheme":
        if variant in EXT_SCHEMES:
            base, fields = EXT_SCHEMES[variant]
            s = cls.make(base, precision)
            for k, v in fields.items():
                setattr(s, k, v)
            return s
        s = cls()
        s.convective_term_solver = FINITE_VOLUME
        s.state_reconstruction = RECON_CHARACTERISTIC
        s.reconstruction_stencil = STENCIL_WENO5
        s.riemann_solver = RIEMANN_HLLC
        s.signal_speed = SIGNAL_SPEED_EINFELDT
        s.flux_splitting = FLUX_SPLITTING_ROE
        s.time_integrator = RK3
        s.precision = precision
        if variant == "fvprim":
            s.state_reconstruction = RECON_PRIMITIVE
        elif variant == "fsroe":
            s.convective_term_solver = FLUX_SPLITTING
        elif variant != "fvchar":
            raise ValueError(variant)
        return s


class Material(C.Structure):
    """alp_material: stiffened gas (gamma, background pressure B, safe variant)."""
    _fields_ = [("gamma", C.c_double), ("background_pressure", C.c_double), ("safe", C.c_int)]

    @classmethod
    def make(cls, gamma: float, B: float = 0.0, safe: bool = False) -> "Material":
        return cls(gamma, B, int(safe))


class CaseCheckpoint(C.Structure):
    """alp_case_checkpoint: what resuming one engine case needs beside its
    neighbour table and blocks."""
    _fields_ = [("dim", C.c_int), ("nb", C.c_int), ("steps", C.c_int), ("max_steps", C.c_int),
                ("t", C.c_double), ("t_end", C.c_double), ("cfl", C.c_double),
                ("cell_size", C.c_double), ("material", Material), ("scheme", Scheme)]


IC_QUADRANTS, IC_BLAST, IC_PROGRAM = 1, 2, 3


class Units(C.Structure):
    """alp_units: UnitHandler references (density, velocity, length)."""
    _fields_ = [("density", C.c_double), ("velocity", C.c_double), ("length", C.c_double)]


class Request(C.Structure):
    """alp_request: one served case (device-evaluated initial condition)."""
    _fields_ = [("dim", C.c_int), ("nblocks", C.c_int * 3), ("periodic", C.c_int * 3),
                ("cell_size", C.c_double), ("material", Material), ("cfl", C.c_double),
                ("t_end", C.c_double), ("max_steps", C.c_int), ("ic_type", C.c_int),
                ("ic_params", C.c_double * 24), ("n_params", C.c_int), ("arrival_s", C.c_double),
                ("h_result", C.POINTER(C.c_double)), ("program", C.c_void_p),
                ("origin", C.c_double * 3), ("units", Units)]


class Result(C.Structure):
    _fields_ = [("arrival_s", C.c_double), ("admitted_s", C.c_double), ("finished_s", C.c_double),
                ("t", C.c_double), ("steps", C.c_int), ("status", C.c_int)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("scheme", Scheme),
                ("max_cases", C.c_int), ("steps_per_poll", C.c_int), ("one_at_a_time", C.c_int),
                ("shortest_first", C.c_int), ("step_set_cells", C.c_double),
                ("abort_file", C.c_char_p)]


_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_V = C.c_void_p
_S = C.c_void_p  # stream
_SIGS = {
    "alp_version": (C.c_char_p, []),
    "alp_last_error": (C.c_char_p, []),
    "alp_scheme_default": (None, [C.POINTER(Scheme)]),
    "alp_convective_fluxes": (C.c_int, [C.c_int, C.POINTER(Scheme), C.POINTER(Material), _V, C.c_int,
                                        C.c_double, _V, _V, _V, _S]),
    "alp_space_rhs_workspace_size": (C.c_size_t, [C.c_int, C.c_int]),
    "alp_space_rhs": (C.c_int, [C.c_int, C.POINTER(Scheme), C.POINTER(Material), _V, C.c_int,
                                C.c_double, _V, _V, C.c_size_t, _S]),
    "alp_space_rhs_static": (C.c_int, [C.c_int, C.POINTER(Scheme), C.POINTER(Material), _V,
                                       C.c_int, C.c_double, _V, _S]),
    "alp_prime_states": (C.c_int, [C.c_int, C.POINTER(Material), _V, C.c_int, _V, _S]),
    "alp_halo_update": (C.c_int, [C.c_int, _V, C.c_int, C.c_int, _V, C.c_int, _S]),
    "alp_timestep_size": (C.c_int, [C.c_int, C.POINTER(Material), _V, C.c_int, C.c_double,
                                    C.c_double, C.c_double, C.c_double, _D, _V, _S]),
    "alp_rk3_stage": (C.c_int, [C.c_int, _V, _V, _V, C.c_int, C.c_int, C.c_double, _S]),
    "alp_engine_create": (C.c_int, [C.c_int, C.POINTER(Scheme), C.c_int, C.c_int, C.POINTER(_V)]),
    "alp_engine_create_elastic": (C.c_int, [C.c_int, C.POINTER(Scheme), C.c_int, C.c_int,
                                            C.POINTER(_V)]),
    "alp_engine_reserve": (C.c_int, [_V, C.c_int]),
    "alp_engine_capacity": (C.c_int, [_V, _I, _I, C.POINTER(C.c_size_t)]),
    "alp_engine_destroy": (C.c_int, [_V]),
    "alp_engine_bytes": (C.c_size_t, [C.c_int, C.c_int, C.c_int]),
    "alp_engine_add_case": (C.c_int, [_V, C.POINTER(Material), C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_int, C.c_int, _I, _D, _I]),
    "alp_engine_add_case_interior": (C.c_int, [_V, C.POINTER(Material), C.c_double, C.c_double,
                                               C.c_double, C.c_double, C.c_int, C.c_int, _I, _D,
                                               _I]),
    "alp_engine_add_case_ic": (C.c_int, [_V, C.POINTER(Material), C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_int, _I, _I, C.c_int, _D, C.c_int, _I]),
    "alp_ic_program_create": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "alp_ic_program_destroy": (None, [_V]),
    "alp_ic_program_info": (C.c_int, [_V, _I, _I, _I]),
    "alp_ic_program_listing": (C.c_int, [_V, C.c_char_p, C.c_int, _I]),
    "alp_ic_evaluate": (C.c_int, [_V, C.c_int, C.c_int, _V, C.c_double, C.POINTER(Units), _V, _S]),
    "alp_engine_add_case_expr": (C.c_int, [_V, C.POINTER(Material), C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.c_int, _I, _I, _D,
                                           C.POINTER(Units), _V, _I]),
    "alp_serve": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(Request), C.c_int, C.POINTER(Result),
                            _D]),
    "alp_engine_remove_case": (C.c_int, [_V, C.c_int]),
    "alp_engine_step": (C.c_int, [_V, C.c_int]),
    "alp_engine_get_case_interior": (C.c_int, [_V, C.c_int, _D, _D, _I]),
    "alp_engine_get_case": (C.c_int, [_V, C.c_int, _D, _D, _I]),
    "alp_engine_all_done": (C.c_int, [_V, _I]),
    "alp_engine_checkpoint_case": (C.c_int, [_V, C.c_int, C.POINTER(CaseCheckpoint), _I, _D]),
    "alp_engine_restore_case": (C.c_int, [_V, C.POINTER(CaseCheckpoint), _I, _D, _I]),
    "alp_engine_stream": (_S, [_V]),
    "alp_engine_set_graph": (C.c_int, [_V, C.c_int]),
    "alp_engine_launches_per_step": (C.c_int, [_V]),
    "alp_engine_launches": (C.c_int, [_V, C.c_int]),
    "alp_engine_path": (C.c_int, [_V]),
    "alp_engine_autotune": (C.c_int, [_V, C.c_int, _I, C.POINTER(C.c_float)]),
    "alp_engine_set_path": (C.c_int, [_V, C.c_int]),
    "alp_levels_create": (C.c_int, [C.c_int, C.POINTER(Scheme), C.POINTER(Material), _I, C.c_double,
                                    C.c_int, _I, _I, C.c_double, C.c_double, C.c_double, C.c_int,
                                    _D, C.POINTER(_V)]),
    "alp_levels_destroy": (C.c_int, [_V]),
    "alp_levels_step": (C.c_int, [_V, C.c_int]),
    "alp_levels_get": (C.c_int, [_V, _D, _D, _I]),
    "alp_levels_info": (C.c_int, [_V, _I, _I, C.POINTER(C.c_longlong), _I]),
    "alp_levels_stream": (_S, [_V]),
    "alp_levels_test_stall_ghosts": (C.c_int, [_V]),
}

# stepping candidates of alp_engine_autotune (ALP_STEP_CANDIDATES)
STEP_CANDIDATES = 6
# the fused tile-stage candidates (16 and 12 warps per CTA)
TILE_CANDIDATES = (4, 5)

_libs = {}


def declared_symbols() -> list[str]:
    """Function names declared in include/alpaca_b200.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(alp_[a-z0-9_]+)\s*\(", text)))


def lib(strict: bool = False) -> C.CDLL:
    """The CUDA library; strict=True loads the build without FMA contraction."""
    if strict not in _libs:
        path = STRICT_LIB_PATH if strict else LIB_PATH
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with "
                              "`python -c 'import __graft_entry__ as g; g.build()'`")
        l = C.CDLL(path)
        for name, (res, args) in _SIGS.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _libs[strict] = l
    return _libs[strict]


def check(rc: int, strict: bool = False) -> None:
    if rc != ALP_OK:
        raise AlpacaError(rc, lib(strict).alp_last_error().decode())
