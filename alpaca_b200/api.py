"""Python face of the C ABI: stateless drop-in calls on device tensors and the
device-resident Engine. torch is used only to hold device memory and streams.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N
from .cases import Case, LevelCase, block_shape

VARIANTS = ("fvchar", "fvprim", "fsroe")


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _stream(stream=None) -> C.c_void_p:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def flux_shape(dim: int, nb: int):
    ne = dim + 2
    return (nb, ne, 17, 17 if dim > 1 else 2, 17 if dim > 2 else 2)


def convective_fluxes(u, dim: int, variant: str, material: N.Material, cell_size: float,
                      precision: int = N.FP64, stream=None, strict: bool = False):
    """ConvectiveTermSolver::UpdateConvectiveFluxes on nb blocks (device tensor
    [nb, ne, TCX, TCY, TCZ] float64). Returns zero-initialised flux arrays with
    the fluxes added, in the reference layout."""
    import torch
    nb = u.shape[0]
    shp = flux_shape(dim, nb)
    f = [torch.zeros(shp, dtype=torch.float64, device=u.device) if d < dim else None
         for d in range(3)]
    sch = N.Scheme.make(variant, precision)
    N.check(N.lib(strict).alp_convective_fluxes(dim, C.byref(sch), C.byref(material), _ptr(u), nb,
                                                cell_size, _ptr(f[0]), _ptr(f[1]), _ptr(f[2]),
                                                _stream(stream)), strict)
    return f


def space_rhs(u, dim: int, variant: str, material: N.Material, cell_size: float,
              precision: int = N.FP64, stream=None, workspace=None, strict: bool = False):
    """SpaceSolver::UpdateFluxes right-hand side (reference layout)."""
    import torch
    nb = u.shape[0]
    rhs = torch.empty_like(u)
    lib = N.lib(strict)
    nbytes = lib.alp_space_rhs_workspace_size(dim, nb)
    if workspace is None:
        workspace = torch.empty(max(nbytes // 8, 1), dtype=torch.float64, device=u.device)
    sch = N.Scheme.make(variant, precision)
    N.check(lib.alp_space_rhs(dim, C.byref(sch), C.byref(material), _ptr(u), nb, cell_size,
                              _ptr(rhs), _ptr(workspace), workspace.numel() * 8,
                              _stream(stream)), strict)
    return rhs


def prime_states(u, dim: int, material: N.Material, stream=None):
    import torch
    p = torch.empty_like(u)
    N.check(N.lib().alp_prime_states(dim, C.byref(material), _ptr(u), u.shape[0], _ptr(p),
                                     _stream(stream)))
    return p


def halo_update(u, dim: int, nbr26, mode: int = N.HALO_ALL, stream=None):
    """In-place halo update; nbr26 is an int32 device tensor [nb, 26]."""
    N.check(N.lib().alp_halo_update(dim, _ptr(u), u.shape[0], u.shape[1], _ptr(nbr26), mode,
                                    _stream(stream)))
    return u


def timestep_size(u, dim: int, material: N.Material, cell_size: float, cfl: float,
                  t: float = 0.0, t_end: float = 1e300, stream=None) -> float:
    import torch
    ws = torch.empty(1, dtype=torch.float64, device=u.device)
    dt = C.c_double()
    N.check(N.lib().alp_timestep_size(dim, C.byref(material), _ptr(u), u.shape[0], cell_size, cfl,
                                      t, t_end, C.byref(dt), _ptr(ws), _stream(stream)))
    return dt.value


def rk3_stage(u, u0, rhs, dim: int, stage: int, dt: float, stream=None):
    N.check(N.lib().alp_rk3_stage(dim, _ptr(u), _ptr(u0), _ptr(rhs), u.shape[0], stage, dt,
                                  _stream(stream)))
    return u


class Engine:
    """Device-resident cases advanced by the fused step (alp_engine_*)."""

    def __init__(self, dim: int, variant: str = "fvchar", precision: int = N.FP64,
                 capacity_blocks: int = 1024, max_cases: int = 64, graph: bool = True,
                 strict: bool = False, elastic: bool = False):
        """elastic: pools reserved for capacity_blocks but backed only by
        reserve() (alp_engine_create_elastic)."""
        self.dim = dim
        self.ne = dim + 2
        self.variant = variant
        self.strict = strict
        self.lib = N.lib(strict)
        # a variant name, or an alp_scheme selection as it is
        sch = variant if isinstance(variant, N.Scheme) else N.Scheme.make(variant, precision)
        h = C.c_void_p()
        create = self.lib.alp_engine_create_elastic if elastic else self.lib.alp_engine_create
        self._check(create(dim, C.byref(sch), capacity_blocks, max_cases, C.byref(h)))
        self.h = h
        self.nb = {}
        if not graph:
            self._check(self.lib.alp_engine_set_graph(self.h, 0))

    def _check(self, rc):
        N.check(rc, self.strict)

    def reserve(self, capacity_blocks: int):
        """Backs exactly that many block slots of an elastic engine."""
        self._check(self.lib.alp_engine_reserve(self.h, capacity_blocks))

    def capacity(self) -> dict:
        cap, used = C.c_int(), C.c_int()
        nbytes = C.c_size_t()
        self._check(self.lib.alp_engine_capacity(self.h, C.byref(cap), C.byref(used),
                                                 C.byref(nbytes)))
        return {"blocks": cap.value, "used": used.value, "bytes": nbytes.value}

    def close(self):
        if getattr(self, "h", None):
            self.lib.alp_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_case(self, case: Case, t0: float = 0.0, max_steps: int | None = None,
                 interior: np.ndarray | None = None) -> int:
        """Adds the case; with `interior` ([nb][NE][16..] interiors, e.g.
        pinned host memory) only those cells are transferred
        (alp_engine_add_case_interior) instead of case.u's full blocks."""
        g = case.grid
        nbr = np.ascontiguousarray(g.nbr26, dtype=np.int32)
        mat = N.Material.make(case.gamma, case.B, False)
        cid = C.c_int()
        steps = case.steps if max_steps is None else max_steps
        if interior is not None:
            assert interior.flags.c_contiguous and interior.dtype == np.float64
            self._check(self.lib.alp_engine_add_case_interior(
                self.h, C.byref(mat), g.cell_size, case.cfl, t0, case.t_end, steps, g.nb,
                nbr.ctypes.data_as(C.POINTER(C.c_int)),
                interior.ctypes.data_as(C.POINTER(C.c_double)), C.byref(cid)))
            self.nb[cid.value] = (g.nb, (g.nb, self.ne) + block_shape(self.dim))
            return cid.value
        u = np.ascontiguousarray(case.u, dtype=np.float64)
        self._check(self.lib.alp_engine_add_case(
            self.h, C.byref(mat), g.cell_size, case.cfl, t0, case.t_end, steps, g.nb,
            nbr.ctypes.data_as(C.POINTER(C.c_int)), u.ctypes.data_as(C.POINTER(C.c_double)),
            C.byref(cid)))
        self.nb[cid.value] = (g.nb, u.shape)
        return cid.value

    def add_case_ic(self, ic_type: int, params, nblocks, cell_size: float, material: N.Material,
                    periodic=(0, 0, 0), cfl: float = 0.6, t_end: float = 1e300,
                    max_steps: int = 0, t0: float = 0.0) -> int:
        """Case with a device-evaluated initial condition on a regular block grid."""
        nbl = (C.c_int * 3)(*(list(nblocks) + [1, 1, 1])[:3])
        per = (C.c_int * 3)(*(list(periodic) + [0, 0, 0])[:3])
        prm = (C.c_double * 24)(*params)
        cid = C.c_int()
        self._check(self.lib.alp_engine_add_case_ic(self.h, C.byref(material), cell_size, cfl, t0,
                                                    t_end, max_steps, nbl, per, ic_type, prm,
                                                    len(params), C.byref(cid)))
        nb = nbl[0] * nbl[1] * nbl[2]
        self.nb[cid.value] = (nb, (nb, self.ne) + block_shape(self.dim))
        return cid.value

    def add_case_expr(self, program: "IcProgram", nblocks, cell_size: float,
                      material: N.Material, periodic=(0, 0, 0), cfl: float = 0.6,
                      t_end: float = 1e300, max_steps: int = 0, t0: float = 0.0,
                      origin=(0.0, 0.0, 0.0), units: N.Units | None = None) -> int:
        """Case whose initial condition is a compiled expression program,
        evaluated on the device over a regular block grid."""
        nbl = (C.c_int * 3)(*(list(nblocks) + [1, 1, 1])[:3])
        per = (C.c_int * 3)(*(list(periodic) + [0, 0, 0])[:3])
        org = (C.c_double * 3)(*(list(origin) + [0.0, 0.0, 0.0])[:3])
        cid = C.c_int()
        self._check(self.lib.alp_engine_add_case_expr(
            self.h, C.byref(material), cell_size, cfl, t0, t_end, max_steps, nbl, per, org,
            C.byref(units) if units is not None else None, program.h, C.byref(cid)))
        nb = nbl[0] * nbl[1] * nbl[2]
        self.nb[cid.value] = (nb, (nb, self.ne) + block_shape(self.dim))
        return cid.value

    def remove_case(self, cid: int):
        self._check(self.lib.alp_engine_remove_case(self.h, cid))
        self.nb.pop(cid, None)

    def step(self, n: int = 1):
        self._check(self.lib.alp_engine_step(self.h, n))

    def get(self, cid: int):
        nb, shp = self.nb[cid]
        out = np.empty(shp, dtype=np.float64)
        t = C.c_double()
        steps = C.c_int()
        self._check(self.lib.alp_engine_get_case(self.h, cid,
                                                 out.ctypes.data_as(C.POINTER(C.c_double)),
                                                 C.byref(t), C.byref(steps)))
        return out, t.value, steps.value

    def get_interior(self, cid: int, out: np.ndarray | None = None):
        """(interiors [nb][NE][16..], t, steps) of case cid
        (alp_engine_get_case_interior); `out` may be a preallocated
        (e.g. pinned) C-contiguous array."""
        nb, _ = self.nb[cid]
        shp = (nb, self.ne) + tuple(16 if d < self.dim else 1 for d in range(3))
        if out is None:
            out = np.empty(shp, dtype=np.float64)
        assert out.shape == shp and out.flags.c_contiguous and out.dtype == np.float64
        t = C.c_double()
        steps = C.c_int()
        self._check(self.lib.alp_engine_get_case_interior(
            self.h, cid, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(t), C.byref(steps)))
        return out, t.value, steps.value

    def checkpoint(self, cid: int) -> dict:
        """The state that resumes case cid exactly (alp_engine_checkpoint_case):
        its blocks, neighbour table, time, step count and settings."""
        nb, shp = self.nb[cid]
        info = N.CaseCheckpoint()
        nbr = np.empty((nb, 26), dtype=np.int32)
        u = np.empty(shp, dtype=np.float64)
        self._check(self.lib.alp_engine_checkpoint_case(
            self.h, cid, C.byref(info), nbr.ctypes.data_as(C.POINTER(C.c_int)),
            u.ctypes.data_as(C.POINTER(C.c_double))))
        return {"dim": info.dim, "steps": info.steps, "max_steps": info.max_steps, "t": info.t,
                "t_end": info.t_end, "cfl": info.cfl, "cell_size": info.cell_size,
                "gamma": info.material.gamma, "background_pressure": info.material.background_pressure,
                "safe": info.material.safe, "scheme": scheme_fields(info.scheme),
                "nbr26": nbr, "blocks": u}

    def restore(self, ck: dict) -> int:
        """Adds the case a checkpoint describes; it continues where it stopped."""
        u = np.ascontiguousarray(ck["blocks"], dtype=np.float64)
        nbr = np.ascontiguousarray(ck["nbr26"], dtype=np.int32)
        info = N.CaseCheckpoint(int(ck["dim"]), u.shape[0], int(ck["steps"]), int(ck["max_steps"]),
                                float(ck["t"]), float(ck["t_end"]), float(ck["cfl"]),
                                float(ck["cell_size"]),
                                N.Material.make(float(ck["gamma"]), float(ck["background_pressure"]),
                                                bool(ck["safe"])),
                                N.Scheme(*[int(v) for v in ck["scheme"]]))
        cid = C.c_int()
        self._check(self.lib.alp_engine_restore_case(
            self.h, C.byref(info), nbr.ctypes.data_as(C.POINTER(C.c_int)),
            u.ctypes.data_as(C.POINTER(C.c_double)), C.byref(cid)))
        self.nb[cid.value] = (u.shape[0], u.shape)
        return cid.value

    def all_done(self) -> bool:
        d = C.c_int()
        self._check(self.lib.alp_engine_all_done(self.h, C.byref(d)))
        return bool(d.value)

    def run_to_end(self, chunk: int = 16, max_chunks: int = 1 << 20):
        for _ in range(max_chunks):
            if self.all_done():
                return
            self.step(chunk)
        raise RuntimeError("engine did not finish")

    def autotune(self, trial_steps: int = 3):
        """Times the stepping candidates on the resident cases (state unchanged)
        and keeps the fastest; returns (chosen index, ms per step per candidate)."""
        chosen = C.c_int()
        ms = (C.c_float * N.STEP_CANDIDATES)()
        self._check(self.lib.alp_engine_autotune(self.h, trial_steps, C.byref(chosen), ms))
        return chosen.value, [float(x) for x in ms]

    def set_path(self, candidate: int):
        self._check(self.lib.alp_engine_set_path(self.h, candidate))

    @property
    def path(self) -> int:
        """The current stepping candidate (numbered as for autotune)."""
        return self.lib.alp_engine_path(self.h)

    @property
    def launches_per_step(self) -> int:
        return self.lib.alp_engine_launches_per_step(self.h)

    def launches(self, n: int) -> int:
        """Kernel launches of one step(n) call."""
        return self.lib.alp_engine_launches(self.h, n)

    @property
    def stream_handle(self) -> int:
        return self.lib.alp_engine_stream(self.h)


class LevelEngine:
    """A multi-level case (alp_levels_*): the leaves of a block tree advanced
    with local time stepping; one CUDA graph per macro step."""

    def __init__(self, case: LevelCase, variant: str = "fvchar", precision: int = N.FP64,
                 max_macro: int = 0, strict: bool = False, t0: float = 0.0):
        self.lib = N.lib(strict)
        self.case, self.variant, self.precision = case, variant, precision
        self.max_macro, self.t0 = max_macro, t0
        self.strict = strict
        self.dim = case.dim
        self.nleaf = case.nleaf
        self.shape = case.u.shape
        sch = N.Scheme.make(variant, precision)
        mat = N.Material.make(case.gamma, case.B)
        level = np.ascontiguousarray(case.level, dtype=np.int32)
        coord = np.ascontiguousarray(case.coord, dtype=np.int32).reshape(-1, 3)
        n0 = np.ascontiguousarray(list(case.n0) + [1] * (3 - len(case.n0)), dtype=np.int32)
        u = np.ascontiguousarray(case.u, dtype=np.float64)
        h = C.c_void_p()
        N.check(self.lib.alp_levels_create(
            case.dim, C.byref(sch), C.byref(mat), n0.ctypes.data_as(N._I), case.h0, case.nleaf,
            level.ctypes.data_as(N._I), coord.ctypes.data_as(N._I), case.cfl, t0, case.t_end,
            max_macro, u.ctypes.data_as(N._D), C.byref(h)), strict)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.alp_levels_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        N.check(self.lib.alp_levels_step(self.h, n), self.strict)

    def get(self):
        """(blocks [nleaf, ne, TC...] with valid interiors, t, macro steps)."""
        out = np.empty(self.shape)
        t = C.c_double()
        m = C.c_int()
        N.check(self.lib.alp_levels_get(self.h, out.ctypes.data_as(N._D), C.byref(t), C.byref(m)),
                self.strict)
        return out, t.value, m.value

    def checkpoint(self) -> dict:
        """The leaves, time and macro steps done (between macro steps nothing
        else carries over: every jump-flux sum has been applied)."""
        u, t, m = self.get()
        return {"blocks": u, "t": t, "macro": m}

    def restore(self, ck: dict, strict: bool = False) -> "LevelEngine":
        """A new level engine for the same tree that continues from ck; the
        macro-step budget counts the steps still to do."""
        c = LevelCase(self.case.name, self.case.dim, self.case.n0, self.case.h0, self.case.level,
                      self.case.coord, ck["blocks"], self.case.gamma, self.case.B, self.case.cfl,
                      self.case.t_end)
        left = self.max_macro - ck["macro"] if self.max_macro > 0 else 0
        if self.max_macro > 0 and left <= 0:
            raise ValueError("the checkpointed case has no macro steps left")
        return LevelEngine(c, self.variant, self.precision, left, strict, ck["t"])

    def info(self) -> dict:
        ng, lm, lp = C.c_int(), C.c_int(), C.c_int()
        cu = C.c_longlong()
        N.check(self.lib.alp_levels_info(self.h, C.byref(ng), C.byref(lm), C.byref(cu),
                                         C.byref(lp)), self.strict)
        return {"ghosts": ng.value, "max_level": lm.value,
                "cell_updates_per_macro_step": cu.value, "launches_per_macro_step": lp.value}

    @property
    def stream_handle(self) -> int:
        return self.lib.alp_levels_stream(self.h) or 0


def serve(requests, hbm_budget_bytes: int, variant: str = "fvchar", precision: int = N.FP64,
          max_cases: int = 256, steps_per_poll: int = 8,
          one_at_a_time: bool = False, keep_results: bool = False, shortest_first: bool = False,
          step_set_cells: float = float(1 << 21), abort_file: str | None = None):
    """Runs the C++ request loop (alp_serve) over a list of serving.Request
    specs. Returns (results as dicts, makespan seconds, final states or None).
    abort_file: once that path exists (checked after every poll) the loop stops
    cleanly; every unfinished request then has status ALP_ABORTED."""
    n = len(requests)
    reqs = (N.Request * n)()
    outs = []
    for i, r in enumerate(requests):
        q = reqs[i]
        q.dim = r.dim
        for d in range(3):
            q.nblocks[d] = r.nblocks[d]
            q.periodic[d] = r.periodic[d]
        q.cell_size = r.cell_size
        q.material = N.Material.make(r.gamma, r.B)
        q.cfl = r.cfl
        q.t_end = r.t_end
        q.max_steps = r.max_steps
        q.ic_type = r.ic_type
        for k, v in enumerate(r.params):
            q.ic_params[k] = v
        q.n_params = len(r.params)
        q.arrival_s = r.arrival_s
        if r.ic_type == N.IC_PROGRAM:
            q.program = r.program.h
            for d in range(3):
                q.origin[d] = r.origin[d]
            if r.units is not None:
                q.units = N.Units(*r.units)
        if keep_results:
            nb = r.nblocks[0] * r.nblocks[1] * r.nblocks[2]
            buf = np.zeros((nb, r.dim + 2) + block_shape(r.dim))
            outs.append(buf)
            q.h_result = buf.ctypes.data_as(C.POINTER(C.c_double))
        else:
            outs.append(None)
    res = (N.Result * n)()
    cfg = N.ServerConfig()
    cfg.hbm_budget_bytes = int(hbm_budget_bytes)
    cfg.scheme = N.Scheme.make(variant, precision)
    cfg.max_cases = max_cases
    cfg.steps_per_poll = steps_per_poll
    cfg.one_at_a_time = int(one_at_a_time)
    cfg.shortest_first = int(shortest_first)
    cfg.step_set_cells = step_set_cells
    cfg.abort_file = abort_file.encode() if abort_file else None
    mk = C.c_double()
    rc = N.lib().alp_serve(C.byref(cfg), reqs, n, res, C.byref(mk))
    if rc not in (N.ALP_OK, N.ALP_ERR_CAPACITY, N.ALP_ABORTED):
        N.check(rc)
    results = [dict(arrival_s=x.arrival_s, admitted_s=x.admitted_s, finished_s=x.finished_s, t=x.t,
                    steps=x.steps, status=x.status) for x in res]
    return results, mk.value, (outs if keep_results else None)


class IcProgram:
    """An initial condition given as expression statements (alp_ic_program_*),
    compiled once on the host; see include/alpaca_b200.h for the language."""

    def __init__(self, text: str, strict: bool = False):
        self.lib = N.lib(strict)
        self.strict = strict
        h = C.c_void_p()
        N.check(self.lib.alp_ic_program_create(text.encode(), C.byref(h)), strict)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.alp_ic_program_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        n, st, nv = C.c_int(), C.c_int(), C.c_int()
        N.check(self.lib.alp_ic_program_info(self.h, C.byref(n), C.byref(st), C.byref(nv)),
                self.strict)
        return {"instructions": n.value, "max_stack": st.value, "variables": nv.value}

    def listing(self) -> list[str]:
        size = 64 * (self.info()["instructions"] + 1)
        buf = C.create_string_buffer(size)
        w = C.c_int()
        N.check(self.lib.alp_ic_program_listing(self.h, buf, size, C.byref(w)), self.strict)
        return buf.value.decode().splitlines()

    def evaluate(self, origins, dim: int, cell_size: float, units: N.Units | None = None,
                 stream=None):
        """Prime states [nb, dim + 2, 16^dim] (non-dimensional) of nodes whose
        origins are the rows of the device tensor origins [nb, 3]."""
        import torch
        nb = origins.shape[0]
        cells = 16 ** dim
        out = torch.empty((nb, dim + 2, cells), dtype=torch.float64, device=origins.device)
        N.check(self.lib.alp_ic_evaluate(self.h, dim, nb, _ptr(origins.contiguous()), cell_size,
                                         C.byref(units) if units is not None else None,
                                         _ptr(out), _stream(stream)), self.strict)
        return out


# Checkpoint files. The reference writes its restart snapshots as HDF5
# (RestartManager::WriteRestartFile, input_output/restart_manager.cpp:301-485):
# group simulation_data with the attributes Time, Dimensions, InternalCells,
# HaloSize and MaximumLevel, and group node_cell_data with the dataset
# Conservatives [node][equation][cells]. These files keep the same names and
# layout in a NumPy archive (no HDF5 library here), plus a case group with what
# resuming a case of this library needs.
_CASE_KEYS = ("steps", "max_steps", "t_end", "cfl", "cell_size", "gamma", "background_pressure",
              "safe")


def scheme_fields(s) -> np.ndarray:
    """The alp_scheme fields in declaration order (int32[8])."""
    return np.array([getattr(s, f) for f, _ in N.Scheme._fields_], dtype=np.int32)


def save_checkpoint(path: str, ck: dict) -> None:
    """Writes one case checkpoint (Engine.checkpoint) to path (.npz)."""
    out = {"simulation_data/Time": np.float64(ck["t"]),
           "simulation_data/Dimensions": np.uint32(ck["dim"]),
           "simulation_data/InternalCells": np.uint32(16),
           "simulation_data/HaloSize": np.uint32(4),
           "simulation_data/MaximumLevel": np.uint32(0),
           "node_cell_data/Conservatives": np.ascontiguousarray(ck["blocks"], dtype=np.float64),
           "case/Neighbours": np.ascontiguousarray(ck["nbr26"], dtype=np.int32),
           "case/Scheme": np.asarray(ck["scheme"], dtype=np.int32)}
    for k in _CASE_KEYS:
        out["case/" + k] = np.asarray(ck[k])
    with open(path, "wb") as f:
        np.savez(f, **out)


def load_checkpoint(path: str) -> dict:
    """Reads a checkpoint file written by save_checkpoint (for Engine.restore)."""
    with np.load(path) as z:
        if int(z["simulation_data/InternalCells"]) != 16 or int(z["simulation_data/HaloSize"]) != 4:
            raise ValueError("checkpoint of another block layout")
        ck = {"t": float(z["simulation_data/Time"]), "dim": int(z["simulation_data/Dimensions"]),
              "blocks": z["node_cell_data/Conservatives"].copy(),
              "nbr26": z["case/Neighbours"].copy()}
        if "case/Scheme" not in z:
            raise ValueError("checkpoint without its scheme selection")
        ck["scheme"] = z["case/Scheme"].copy()
        for k in _CASE_KEYS:
            v = z["case/" + k]
            ck[k] = v.item()
    return ck
