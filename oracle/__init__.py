"""CPU oracles for the ALPACA block right-hand side (TEST INFRASTRUCTURE ONLY).

Two independent implementations of the same path, used only by ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU arm, always as the checker of
the CUDA path and never as the thing measured or shipped:

* :class:`Restatement` - ``oracle/alpaca_oracle.c``, a plain-C restatement of
  the reference (tumaer/ALPACA) hot path, built to ``oracle/_build/liboracle.so``.
* :class:`Reference` - ALPACA's own sources compiled in place by
  ``oracle/Makefile`` into ``oracle/_ref/libalpref_d<D>_<variant>.so`` (absent
  when the reference sources were not available at build time).

Both expose the same methods on numpy arrays in the reference's block layout:
``u[nb, ne, TCX, TCY, TCZ]`` (TC = 24 in active, 1 in inactive dimensions).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "liboracle.so")
# the same restatement with every double replaced by an operation-counting scalar
OPCOUNT_SO = os.path.join(HERE, "_build", "liboracle_ops.so")
REF_DIR = os.path.join(HERE, "_ref")

FLUX_SPLITTING, FINITE_VOLUME = 0, 1
RECON_CONSERVATIVE, RECON_PRIMITIVE, RECON_CHARACTERISTIC = 0, 1, 2

# variant name -> (solver, reconstruction), as selected in the reference's
# user_specifications/riemann_solver_settings.h and state_reconstruction_settings.h
VARIANTS = {
    "fvchar": (FINITE_VOLUME, RECON_CHARACTERISTIC),
    "fvprim": (FINITE_VOLUME, RECON_PRIMITIVE),
    "fsroe": (FLUX_SPLITTING, RECON_CHARACTERISTIC),
}

# Further selections: name -> (base variant, (stencil, riemann solver, signal
# speed, flux splitting)) with the values of the reference's enums.
WENO5, WENO5Z, TENO5, WENO3, FIRST_ORDER, WENO7 = 4, 7, 11, 1, 0, 13
HLLC, HLLC_LM, HLL = 0, 1, 2
EINFELDT, DAVIS, TORO, ARITHMETIC = 0, 1, 2, 3
ROE, LLF, GLF, ROE_M, LLF_M = 0, 1, 2, 3, 4
RK2, RK3 = 0, 1  # TimeIntegrators (numerical_setup.h:26)
DEFAULT_OPTIONS = (WENO5, HLLC, EINFELDT, ROE, RK3)
EXT_VARIANTS = {
    "fvchar_weno5z": ("fvchar", (WENO5Z, HLLC, EINFELDT, ROE)),
    "fvchar_teno5": ("fvchar", (TENO5, HLLC, EINFELDT, ROE)),
    "fvchar_weno3": ("fvchar", (WENO3, HLLC, EINFELDT, ROE)),
    "fvchar_first": ("fvchar", (FIRST_ORDER, HLLC, EINFELDT, ROE)),
    "fvchar_hll": ("fvchar", (WENO5, HLL, EINFELDT, ROE)),
    "fvchar_hllclm": ("fvchar", (WENO5, HLLC_LM, EINFELDT, ROE)),
    "fvchar_davis": ("fvchar", (WENO5, HLLC, DAVIS, ROE)),
    "fvchar_toro": ("fvchar", (WENO5, HLLC, TORO, ROE)),
    "fvchar_arith": ("fvchar", (WENO5, HLLC, ARITHMETIC, ROE)),
    "fvprim_teno5": ("fvprim", (TENO5, HLLC, EINFELDT, ROE)),
    "fs_llf": ("fsroe", (WENO5, HLLC, EINFELDT, LLF)),
    "fs_roem": ("fsroe", (WENO5, HLLC, EINFELDT, ROE_M)),
    "fs_llfm": ("fsroe", (WENO5, HLLC, EINFELDT, LLF_M)),
    "fs_teno5": ("fsroe", (TENO5, HLLC, EINFELDT, ROE)),
    # the four single-phase selections of the reference testsuite's DetailedSod
    # table (32-cell blocks, RK3) that differ from the defaults in two places
    "fvchar_weno3_hll": ("fvchar", (WENO3, HLL, EINFELDT, ROE)),
    "fs_weno3": ("fsroe", (WENO3, HLLC, EINFELDT, ROE)),
    "fs_llf_weno3": ("fsroe", (WENO3, HLLC, EINFELDT, LLF)),
    "fs_llfm_weno3": ("fsroe", (WENO3, HLLC, EINFELDT, LLF_M)),
    # global Lax-Friedrichs (maxima over all blocks of the call / case)
    "fs_glf": ("fsroe", (WENO5, HLLC, EINFELDT, GLF)),
    "fs_glf_weno5z": ("fsroe", (WENO5Z, HLLC, EINFELDT, GLF)),
    # TVD-RK2 selections of the DetailedSod table (fifth option: time integrator)
    "rk2_fvchar_weno3": ("fvchar", (WENO3, HLLC, EINFELDT, ROE, RK2)),
    "rk2_fvchar_hll_weno5z": ("fvchar", (WENO5Z, HLL, EINFELDT, ROE, RK2)),
    "rk2_fs_glf": ("fsroe", (WENO5, HLLC, EINFELDT, GLF, RK2)),
    "rk2_fs_llf_weno5z": ("fsroe", (WENO5Z, HLLC, EINFELDT, LLF, RK2)),
    "rk2_fs_roem_weno3": ("fsroe", (WENO3, HLLC, EINFELDT, ROE_M, RK2)),
    "rk2_fs_llfm": ("fsroe", (WENO5, HLLC, EINFELDT, LLF_M, RK2)),
    "rk2_fs_llfm_weno5z": ("fsroe", (WENO5Z, HLLC, EINFELDT, LLF_M, RK2)),
    # WENO7 (8-cell stencils) and the WENO7 rows of the DetailedSod table
    "fvchar_weno7": ("fvchar", (WENO7, HLLC, EINFELDT, ROE)),
    "fs_roem_weno7": ("fsroe", (WENO7, HLLC, EINFELDT, ROE_M)),
    "rk2_fvchar_weno7": ("fvchar", (WENO7, HLLC, EINFELDT, ROE, RK2)),
    "rk2_fs_glf_weno7": ("fsroe", (WENO7, HLLC, EINFELDT, GLF, RK2)),
    "rk2_fs_weno7": ("fsroe", (WENO7, HLLC, EINFELDT, ROE, RK2)),
}


def variant_spec(variant: str):
    """(solver, reconstruction, options) of a variant name."""
    if variant in VARIANTS:
        return VARIANTS[variant] + (DEFAULT_OPTIONS,)
    base, opts = EXT_VARIANTS[variant]
    return VARIANTS[base] + (tuple(opts) + DEFAULT_OPTIONS[len(opts):],)

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)


def build(quiet: bool = True) -> None:
    """Build both oracles (make -C oracle); the reference part needs its sources."""
    out = subprocess.run(["make", "-C", HERE, "-j", str(os.cpu_count() or 4), "all"],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    if not quiet:
        print(out.stdout[-2000:])


def geometry(dim: int):
    tc = tuple(24 if d < dim else 1 for d in range(3))
    ic = tuple(16 if d < dim else 1 for d in range(3))
    return tc, ic


class _Common:
    dim: int
    ne: int

    def _shapes(self, nb):
        tc, ic = geometry(self.dim)
        return (nb, self.ne) + tc, (nb, self.ne) + tuple(n + 1 for n in ic)


def _prediction(fn, parent, octant, start, count, child):
    parent = np.ascontiguousarray(parent, dtype=np.float64)
    child = np.zeros_like(parent) if child is None else np.ascontiguousarray(child, dtype=np.float64)
    st = np.zeros(3, dtype=np.int32)
    ct = np.zeros(3, dtype=np.int32)
    st[:len(start)] = start
    ct[:len(count)] = count
    if fn(_dp(parent), int(octant), st.ctypes.data_as(_I), ct.ctypes.data_as(_I), _dp(child)):
        raise ValueError("prediction: bad range")
    return child


def _load(path: str):
    """Loads a build of alpaca_oracle.c and declares its entry points."""
    lib = C.CDLL(path)
    lib.oracle_weno5.argtypes = [_D, _D, _D]
    lib.oracle_eos.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, _D, _D, _D]
    lib.oracle_prime_states.argtypes = [C.c_int, _D, C.c_int, C.c_double, C.c_double, C.c_int, _D]
    lib.oracle_space_rhs.argtypes = [C.c_int, C.c_int, C.c_int, _D, C.c_int, C.c_double,
                                     C.c_double, C.c_int, C.c_double, _D, _D, _D, _D, C.c_int]
    lib.oracle_timestep.argtypes = [C.c_int, _D, C.c_int, C.c_double, C.c_double, C.c_int,
                                    C.c_double, C.c_double, C.c_double, C.c_double, _D]
    lib.oracle_halo_fill.argtypes = [C.c_int, _D, C.c_int, C.c_int, _I, C.c_int, C.c_int]
    lib.oracle_halo_update.argtypes = [C.c_int, _D, C.c_int, _I]
    lib.oracle_run.argtypes = [C.c_int, C.c_int, C.c_int, _D, C.c_int, _I, C.c_double,
                               C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
                               C.c_int, C.c_int, _D, _I, _D]
    lib.oracle_set_options.argtypes = [C.c_int] * 4
    lib.oracle_prediction.argtypes = [C.c_int, _D, C.c_int, _I, _I, _D]
    lib.oracle_set_time_integrator.argtypes = [C.c_int]
    lib.oracle_level_halos.argtypes = [C.c_int, _D, C.c_int, _I, _I, _I]
    lib.oracle_levels_run.argtypes = [C.c_int, C.c_int, C.c_int, _D, C.c_int, _I, _I, _I,
                                      C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                      C.c_double, C.c_int, C.c_int, _D, _I, _D]
    return lib


class Restatement(_Common):
    """The plain-C restatement, for one dimension and scheme variant."""

    _lib = None
    _path = RESTATEMENT_SO

    def __init__(self, dim: int, variant: str = "fvchar"):
        cls = type(self)
        if cls._lib is None:
            if not os.path.exists(cls._path):
                build()
            cls._lib = _load(cls._path)
        self.lib = cls._lib
        self.dim = dim
        self.ne = dim + 2
        self.variant = variant
        self.solver, self.recon, self.options = variant_spec(variant)
        # every entry point below reads the process-wide selection: set it first
        self._select()

    def _select(self):
        if self.lib.oracle_set_options(*self.options[:4]) or \
                self.lib.oracle_set_time_integrator(self.options[4]):
            raise ValueError(f"unknown options {self.options}")

    # -- scalar kernels --
    def weno5(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        l, r = C.c_double(), C.c_double()
        self.lib.oracle_weno5(_dp(v), C.byref(l), C.byref(r))
        return l.value, r.value

    def eos(self, gamma, B, safe, cons, prim):
        cons = np.ascontiguousarray(cons, dtype=np.float64)
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        out = np.zeros(6)
        self.lib.oracle_eos(self.dim, gamma, B, int(safe), _dp(cons), _dp(prim), _dp(out))
        return out

    def prediction(self, parent, octant, start, count, child=None):
        """Multiresolution::Prediction of one field buffer (tc shape) into the
        child cells start .. start + count of a child at position octant."""
        return _prediction(lambda *a: self.lib.oracle_prediction(self.dim, *a),
                           parent, octant, start, count, child)

    # -- block kernels --
    def prime_states(self, u, gamma, B=0.0, safe=False):
        u = np.ascontiguousarray(u, dtype=np.float64)
        p = np.empty_like(u)
        self.lib.oracle_prime_states(self.dim, _dp(u), u.shape[0], gamma, B, int(safe), _dp(p))
        return p

    def space_rhs(self, u, gamma, B, safe, cell_size, nthreads=1):
        """Returns (fx, fy, fz, rhs) for blocks whose halos are filled."""
        self._select()
        u = np.ascontiguousarray(u, dtype=np.float64)
        nb = u.shape[0]
        _, fshape = self._shapes(nb)
        fx, fy, fz = (np.zeros(fshape) for _ in range(3))
        rhs = np.zeros_like(u)
        rc = self.lib.oracle_space_rhs(self.dim, self.solver, self.recon, _dp(u), nb, gamma, B,
                                       int(safe), cell_size, _dp(fx), _dp(fy), _dp(fz), _dp(rhs),
                                       nthreads)
        if rc:
            raise RuntimeError(f"oracle_space_rhs rc={rc}")
        return fx, fy, fz, rhs

    def timestep(self, u, gamma, B, safe, cell_size, cfl, t=0.0, t_end=1e300):
        u = np.ascontiguousarray(u, dtype=np.float64)
        dt = C.c_double()
        self.lib.oracle_timestep(self.dim, _dp(u), u.shape[0], gamma, B, int(safe), cell_size, cfl,
                                 t, t_end, C.byref(dt))
        return dt.value

    def halo_fill(self, u, nbr26, faces_only=False, zero_gradient=False):
        """In-place same-level halo copy over 26 (or 2*dim face) regions, then
        optionally the zero-gradient slabs of domain faces."""
        assert u.dtype == np.float64 and u.flags.c_contiguous
        nbr26 = np.ascontiguousarray(nbr26, dtype=np.int32)
        self.lib.oracle_halo_fill(self.dim, _dp(u), u.shape[0], u.shape[1], _ip(nbr26),
                                  int(faces_only), int(zero_gradient))
        return u

    def halo_update(self, u, nbr):
        """In-place six-face halo copy plus zero-gradient slabs on domain faces."""
        assert u.dtype == np.float64 and u.flags.c_contiguous
        nbr = np.ascontiguousarray(nbr, dtype=np.int32)
        self.lib.oracle_halo_update(self.dim, _dp(u), u.shape[0], _ip(nbr))
        return u

    def run(self, u, nbr, gamma, B, safe, cell_size, cfl, t_end, max_steps=0, t0=0.0,
            nthreads=1):
        """Single-level time loop. Returns (u_final, t, steps, dt_log)."""
        self._select()
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        nbr = np.ascontiguousarray(nbr, dtype=np.int32)
        cap = max_steps if max_steps > 0 else 1000000
        dts = np.zeros(cap)
        t = C.c_double(t0)
        steps = C.c_int()
        rc = self.lib.oracle_run(self.dim, self.solver, self.recon, _dp(u), u.shape[0], _ip(nbr),
                                 gamma, B, int(safe), cell_size, cfl, t_end, max_steps, nthreads,
                                 C.byref(t), C.byref(steps), _dp(dts))
        if rc:
            raise RuntimeError(f"oracle_run rc={rc}")
        return u, t.value, steps.value, dts[: steps.value].copy()

    def level_halos(self, u, level, coord, n0):
        """The leaves' face halos of one multi-level snapshot, as a stage of
        the level step fills them (oracle_level_halos); returns a copy of u."""
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        level = np.ascontiguousarray(level, dtype=np.int32)
        coord = np.ascontiguousarray(coord, dtype=np.int32).reshape(-1, 3)
        n0 = np.ascontiguousarray(list(n0) + [1] * (3 - len(n0)), dtype=np.int32)
        rc = self.lib.oracle_level_halos(self.dim, _dp(u), u.shape[0], _ip(level), _ip(coord),
                                         _ip(n0))
        if rc:
            raise RuntimeError(f"oracle_level_halos rc={rc}")
        return u

    def levels_run(self, u, level, coord, n0, h0, gamma, B, safe, cfl, t_end, max_macro=0,
                   t0=0.0, nthreads=1):
        """Multi-level time loop with local time stepping (leaves of a block
        tree). Returns (u_final, t, macro_steps, micro_dt_log)."""
        self._select()
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        level = np.ascontiguousarray(level, dtype=np.int32)
        coord = np.ascontiguousarray(coord, dtype=np.int32).reshape(-1, 3)
        n0 = np.ascontiguousarray(list(n0) + [1] * (3 - len(n0)), dtype=np.int32)
        nmicro = 1 << int(level.max())
        cap = (max_macro if max_macro > 0 else 100000) * nmicro
        dts = np.zeros(cap)
        t = C.c_double(t0)
        macro = C.c_int()
        rc = self.lib.oracle_levels_run(self.dim, self.solver, self.recon, _dp(u), u.shape[0],
                                        _ip(level), _ip(coord), _ip(n0), h0, gamma, B, int(safe),
                                        cfl, t_end, max_macro, nthreads, C.byref(t),
                                        C.byref(macro), _dp(dts))
        if rc:
            raise RuntimeError(f"oracle_levels_run rc={rc}")
        return u, t.value, macro.value, dts[: macro.value * nmicro].copy()


class OpCounting(Restatement):
    """The restatement compiled with an operation-counting scalar
    (oracle/flop_count.cpp): same results, plus the floating-point operations
    the reference algorithm executes. Single-threaded (nthreads must stay 1)."""

    _lib = None
    _path = OPCOUNT_SO
    FIELDS = ("add", "mul", "div", "sqrt", "cmp", "abs", "pow", "sin")

    def __init__(self, dim: int, variant: str = "fvchar"):
        super().__init__(dim, variant)
        self.lib.oracle_op_counts.argtypes = [C.POINTER(C.c_longlong)]
        self.lib.oracle_op_reset.argtypes = []

    def reset(self) -> None:
        self.lib.oracle_op_reset()

    def counts(self) -> dict:
        out = (C.c_longlong * 8)()
        self.lib.oracle_op_counts(out)
        return dict(zip(self.FIELDS, (int(x) for x in out)))


class Reference(_Common):
    """ALPACA's own hot-path code (oracle/_ref), one library per dimension and variant."""

    _libs: dict = {}

    @staticmethod
    def available(dim: int = 3, variant: str = "fvchar") -> bool:
        return os.path.exists(os.path.join(REF_DIR, f"libalpref_d{dim}_{variant}.so"))

    def __init__(self, dim: int, variant: str = "fvchar"):
        key = (dim, variant)
        path = os.path.join(REF_DIR, f"libalpref_d{dim}_{variant}.so")
        if key not in Reference._libs:
            if not os.path.exists(path):
                raise FileNotFoundError(path)
            lib = C.CDLL(path)
            lib.ref_config.argtypes = [_I] * 5
            lib.ref_weno5.argtypes = [_D, _D, _D]
            lib.ref_eos.argtypes = [C.c_double, C.c_double, C.c_int, _D, _D, _D]
            lib.ref_prime_states.argtypes = [_D, C.c_int, C.c_double, C.c_double, C.c_int, _D]
            lib.ref_space_rhs.argtypes = [_D, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double,
                                          _D, _D, _D, _D, C.c_int]
            lib.ref_run.argtypes = [_D, C.c_int, _I, C.c_double, C.c_double, C.c_int, C.c_double,
                                    C.c_double, C.c_double, C.c_int, C.c_int, _D, _I, _D]
            lib.ref_prediction.argtypes = [_D, C.c_int, _I, _I, _D]
            Reference._libs[key] = lib
        self.lib = Reference._libs[key]
        vals = [C.c_int() for _ in range(5)]
        self.lib.ref_config(*[C.byref(v) for v in vals])
        self.dim, self.ne = vals[0].value, vals[1].value
        assert self.dim == dim
        self.variant = variant

    def weno5(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        l, r = C.c_double(), C.c_double()
        self.lib.ref_weno5(_dp(v), C.byref(l), C.byref(r))
        return l.value, r.value

    def prediction(self, parent, octant, start, count, child=None):
        return _prediction(self.lib.ref_prediction, parent, octant, start, count, child)

    def eos(self, gamma, B, safe, cons, prim):
        cons = np.ascontiguousarray(cons, dtype=np.float64)
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        out = np.zeros(6)
        self.lib.ref_eos(gamma, B, int(safe), _dp(cons), _dp(prim), _dp(out))
        return out

    def prime_states(self, u, gamma, B=0.0, safe=False):
        u = np.ascontiguousarray(u, dtype=np.float64)
        p = np.empty_like(u)
        self.lib.ref_prime_states(_dp(u), u.shape[0], gamma, B, int(safe), _dp(p))
        return p

    def space_rhs(self, u, gamma, B, safe, cell_size, nthreads=1):
        u = np.ascontiguousarray(u, dtype=np.float64)
        nb = u.shape[0]
        _, fshape = self._shapes(nb)
        fx, fy, fz = (np.zeros(fshape) for _ in range(3))
        rhs = np.zeros_like(u)
        self.lib.ref_space_rhs(_dp(u), nb, gamma, B, int(safe), cell_size, _dp(fx), _dp(fy),
                               _dp(fz), _dp(rhs), nthreads)
        return fx, fy, fz, rhs

    def run(self, u, nbr, gamma, B, safe, cell_size, cfl, t_end, max_steps=0, t0=0.0,
            nthreads=1):
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        nbr = np.ascontiguousarray(nbr, dtype=np.int32)
        cap = max_steps if max_steps > 0 else 1000000
        dts = np.zeros(cap)
        t = C.c_double(t0)
        steps = C.c_int()
        self.lib.ref_run(_dp(u), u.shape[0], _ip(nbr), gamma, B, int(safe), cell_size, cfl, t_end,
                         max_steps, nthreads, C.byref(t), C.byref(steps), _dp(dts))
        return u, t.value, steps.value, dts[: steps.value].copy()


class Glue:
    """ALPACA's own multi-level glue (TopologyManager, Tree, Averager,
    InternalHaloManager) on one rank, 3D: oracle/_ref/libalpglue_d3.so."""

    _lib = None
    path = os.path.join(REF_DIR, "libalpglue_d3.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.path)

    def __init__(self):
        cls = type(self)
        if cls._lib is None:
            lib = C.CDLL(cls.path)
            lib.glue_level_halos.restype = C.c_int
            lib.glue_level_halos.argtypes = [_D, C.c_int, _I, _I, _I]
            lib.glue_last_error.restype = C.c_char_p
            cls._lib = lib
        self.lib = cls._lib

    def level_halos(self, u, level, coord, n0):
        """Every leaf's buffer after the reference's averaging and level-by-
        level halo update of one snapshot (levels_glue_harness.cpp)."""
        u = np.array(u, dtype=np.float64, order="C", copy=True)
        level = np.ascontiguousarray(level, dtype=np.int32)
        coord = np.ascontiguousarray(coord, dtype=np.int32).reshape(-1, 3)
        n0 = np.ascontiguousarray(list(n0) + [1] * (3 - len(n0)), dtype=np.int32)
        if self.lib.glue_level_halos(_dp(u), u.shape[0], _ip(level), _ip(coord), _ip(n0)):
            raise RuntimeError(self.lib.glue_last_error().decode())
        return u
