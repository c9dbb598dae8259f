"""Benchmark of the block RHS + SSP-RK3 engine on the 3D periodic 128^3 case.

Workload (the headline configuration): 8 x 8 x 8 = 512 blocks of 16^3 cells
(128^3 cells, 4-cell halos), ideal gas gamma 1.4, seeded Fourier-mode fields
with a planar Mach-2 Rankine-Hugoniot shock, WENO5-JS characteristic
reconstruction + HLLC (Einfeldt) + SSP-RK3 at CFL 0.6, all FP64.
One step = one full SSP-RK3 step of the whole domain (dt reduction, three
stages of fluxes / divergence + stage update / halo fill).
metric: cell-updates/s = interior cells x steps / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank advances its own copy of the case (replicas: the path
does not shard across GPUs); value = cells x steps x N / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
B_ALG_3D = 320.0  # algorithmic HBM bytes per 3D cell-update (64 * N_eq, FP64 state)
# Floating-point operations (add + mul + div + sqrt) of the reference algorithm
# per 3D cell-update (one full SSP-RK3 step incl. prime states and dt), counted
# by the operation-counting build of the oracle on a seeded one-block case;
# tests/test_oracle.py::test_op_counts_match_bench_constants re-counts them.
FLOPS_PER_CELL_UPDATE_3D = {"fvchar": 15767, "fvprim": 10192, "fsroe": 22478}
FLOPS_PER_CELL_UPDATE_2D = {"fvchar": 8004, "fvprim": 5448, "fsroe": 10605}
# DRAM bytes per SSP-RK3 step of the 128^3 workload (sum of dram__bytes_read.sum
# and dram__bytes_write.sum over the step's kernels, one ncu capture; summary in
# profiles/step_fvchar_128cubed.md)
TRAFFIC_PER_STEP = {("fvchar", "fp64"): 4.359e9}
# DRAM bytes per cell-update of the multi-level step (fvchar, FP64): one ncu
# capture of a macro step of the same hierarchy at n0 = 2 (31 / 264 leaves, 176
# ghosts, 4.58 M cell-updates, 9.38 GB), scaled by cell-updates (summary in
# profiles/levels_3d_spherical_shock.md)
LEVELS_DRAM_PER_CELL_UPDATE = {("fvchar", "fp64"): 2048.0}
# stepping candidates of alp_engine_autotune, in its numbering
CANDIDATES = ["face fluxes, 128-thread blocks", "face fluxes, 64-thread blocks", "pencil sweeps",
              "face fluxes and stage updates overlapped in batches",
              "fused tile stages (TMA-staged, one persistent launch), 16 warps",
              "fused tile stages (TMA-staged, one persistent launch), 12 warps"]


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--variant", default="fvchar", choices=["fvchar", "fvprim", "fsroe"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                   help="fp32: FP32 reconstruction/Riemann arithmetic, FP64 state")
    p.add_argument("--blocks", type=int, default=8, help="blocks per dimension")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--serving-requests", type=int, default=32)
    p.add_argument("--step-set-cells", type=float, default=float(1 << 21),
                   help="cells stepping together under shortest-remaining-work-first serving")
    p.add_argument("--precision-report", action="store_true",
                   help="FP32-flux vs FP64 errors per field after 200 steps (128^3, 256^3, water)")
    p.add_argument("--serving-only", action="store_true",
                   help="run only the serving comparison and print its JSON")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the FP32-flux and multi-level entries of the default line")
    p.add_argument("--path", type=int, default=None,
                   help="stepping candidate to use instead of the autotuner's choice "
                        "(numbered as alp_engine_autotune; for profiling one path)")
    p.add_argument("--levels", action="store_true",
                   help="multi-level batching: 3-level spherical-shock hierarchy with local "
                        "time stepping (one line; steps are macro steps)")
    p.add_argument("--levels-n0", type=int, default=4,
                   help="level-0 nodes per dimension of that hierarchy (4: 8 / 294 / 1232 "
                        "leaves; 2, a small case for profiling: 0 / 31 / 264)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: through
    NVML every 5 ms (the GPU found by its PCI bus id, so a restricted device
    list maps correctly), one sample taken before the region starts and one as
    it ends; nvidia-smi every 100 ms when NVML is unavailable."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def _nvml_sample(self):
        n = self.nvml
        sm = n.nvmlDeviceGetClockInfo(self.h, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(self.h, n.NVML_CLOCK_SM)
        r = n.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        flag = lambda bit: "Active" if r & bit else "Not Active"
        self.rows.append([str(self.index), str(sm), str(mx), "", hex(r),
                          flag(n.nvmlClocksEventReasonHwSlowdown),
                          flag(n.nvmlClocksEventReasonHwThermalSlowdown),
                          flag(n.nvmlClocksEventReasonSwThermalSlowdown),
                          flag(n.nvmlClocksEventReasonSwPowerCap)])

    def _nvml_loop(self):
        while not self.stop.wait(0.005):
            try:
                self._nvml_sample()
            except Exception:
                return

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            try:
                import torch
                pr = torch.cuda.get_device_properties(self.index)
                bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
                self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.nvml = pynvml
            self._nvml_sample()
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.nvml:
            try:
                self._nvml_sample()
            except Exception:
                pass
            self.stop.set()
            self.thread.join(timeout=1)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            return
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = []
        mx = None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except Exception:
                pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def max_over_ranks(x: float, ws: int, dev=None) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=dev if dev is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int, dev=None):
    if ws > 1:
        import torch.distributed as dist
        if dev is not None:
            dist.barrier(device_ids=[dev.index])
        else:
            dist.barrier()


# ---------------------------------------------------------------------------
# CPU arm: the reference's own hot path (oracle/_ref) on the host cores
# ---------------------------------------------------------------------------

def reference_cpu_sample(variant: str, budget_s: float, nthreads: int, steps: int | None = None,
                         warmup: int = 0, nblocks: int = 8):
    """Times the reference's compiled code (oracle/_ref; the restatement when the
    reference was not built) on the bench workload itself: the periodic 8x8x8-
    block (128^3-cell) Fourier + Mach-2 case, all blocks of every step (the
    reference parallelises over blocks; here host threads over blocks). With
    steps None, as many steps as fit in about budget_s seconds."""
    import oracle
    from alpaca_b200 import cases
    kind = "reference" if oracle.Reference.available(3, variant) else "port"
    impl = oracle.Reference(3, variant) if kind == "reference" else oracle.Restatement(3, variant)
    case = cases.fourier_shock(nblocks, dim=3, seed=1)
    g = case.grid
    u = case.u
    if warmup:
        u = impl.run(u, g.nbr, case.gamma, 0.0, False, g.cell_size, case.cfl, 1e300,
                     max_steps=warmup, nthreads=nthreads)[0]
    if steps is None:
        t0 = time.perf_counter()
        u = impl.run(u, g.nbr, case.gamma, 0.0, False, g.cell_size, case.cfl, 1e300, max_steps=1,
                     nthreads=nthreads)[0]
        one = time.perf_counter() - t0
        steps = max(1, int(budget_s / max(one, 1e-3)))
    t0 = time.perf_counter()
    impl.run(u, g.nbr, case.gamma, 0.0, False, g.cell_size, case.cfl, 1e300, max_steps=steps,
             nthreads=nthreads)
    dt = time.perf_counter() - t0
    cells = g.nb * 4096
    side = nblocks * 16
    return {"value": cells * steps / dt, "unit": METRIC, "cores": nthreads, "kind": kind,
            "sample": f"{steps} SSP-RK3 steps of the {nblocks}x{nblocks}x{nblocks}-block "
                      f"({side}^3-cell) periodic Fourier + Mach-2 workload, {variant}, FP64, "
                      f"{nthreads} threads",
            "seconds": dt, "steps": steps, "blocks": g.nb}


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return
    n = os.cpu_count() or 1
    r = reference_cpu_sample(args.variant, 0.0, n, steps=args.steps, warmup=args.warmup,
                             nblocks=args.blocks)
    line = {"metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["seconds"] * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "3d_periodic_fourier_mach2_128cubed", "variant": args.variant,
                       "blocks": r["blocks"], "cells": r["blocks"] * 4096},
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def fp64_peak():
    lib = C.CDLL(os.path.join(ROOT, "alpaca_b200", "libalpaca_b200_probe.so"))
    lib.alp_probe_fp64_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    v = C.c_double()
    if lib.alp_probe_fp64_peak(20000, 8, C.byref(v)) != 0:
        return None
    return v.value


def serving_bound(reqs, one_at_a_time_makespan_s, fp64_tflops, engine_3d_rate=None):
    """Lower bound on the makespan of a request stream: the FP64 operations of
    all its cell-updates (the reference algorithm's count per 2D / 3D
    cell-update, FV characteristic) at the measured FP64 peak, and the last
    arrival. Against the one-at-a-time makespan it bounds the cases/s gain any
    batching can reach, and gives the throughput a 3x gain would need. With
    the engine's measured 3D FP64 rate, also the time its 3D work alone takes
    at that rate (a floor for this engine, 2D work not counted)."""
    flops = sum(r.blocks * 16 ** r.dim * r.max_steps *
                (FLOPS_PER_CELL_UPDATE_3D if r.dim == 3 else FLOPS_PER_CELL_UPDATE_2D)["fvchar"]
                for r in reqs)
    cu = sum(r.blocks * 16 ** r.dim * r.max_steps for r in reqs)
    work_floor = flops / (fp64_tflops * 1e12) if fp64_tflops else None
    last = max(r.arrival_s for r in reqs)
    floor = max(work_floor or 0.0, last)
    cu3 = sum(r.blocks * 16 ** r.dim * r.max_steps for r in reqs if r.dim == 3)
    engine = None
    if engine_3d_rate:
        floor_e = max(cu3 / engine_3d_rate, last)
        engine = {"cell_updates_3d": int(cu3), "rate_3d_fp64": engine_3d_rate,
                  "floor_makespan_s": floor_e,
                  "max_cases_per_s_vs_one_at_a_time": one_at_a_time_makespan_s / floor_e}
    return {"cell_updates": int(cu), "fp64_operations": float(flops),
            "fp64_peak_tflops": fp64_tflops, "work_floor_makespan_s": work_floor,
            "last_arrival_s": last, "floor_makespan_s": floor,
            "one_at_a_time_makespan_s": one_at_a_time_makespan_s,
            "max_cases_per_s_vs_one_at_a_time": one_at_a_time_makespan_s / floor,
            "three_x_reachable_in_fp64": one_at_a_time_makespan_s / floor >= 3.0,
            "cell_updates_per_s_needed_for_3x": 3.0 * cu / one_at_a_time_makespan_s,
            "engine": engine}


def serving_report(args, engine_3d_rate=None):
    """Serving form: seeded request streams (2D four-quadrant problems and 3D
    gas / water blasts, log-uniform 4-2048 blocks, 200-2000 steps, Poisson
    arrivals at 10, 50 and 200 requests/s) served one case at a time in FP64,
    and with continuous batching in FP64 and in the FP32-flux form (at 50/s also
    shortest remaining work first, --step-set-cells stepping together); time-
    to-solution percentiles and cases/s per mode, and the work bound of each
    stream (serving_bound)."""
    import numpy as np

    from alpaca_b200 import api, serving
    from alpaca_b200 import native as N
    budget = 160 << 30
    fp64 = fp64_peak()
    base_modes = (("one_at_a_time_fp64", N.FP64, True, False), ("batched_fp64", N.FP64, False, False),
                  ("batched_fp32_flux", N.FP32_FLUX, False, False))
    srpt_modes = (("batched_shortest_first_fp64", N.FP64, False, True),
                  ("batched_shortest_first_fp32_flux", N.FP32_FLUX, False, True))

    def serve_stream(rate, modes):
        reqs = serving.request_stream(args.serving_requests, seed=11, rate_hz=rate)
        out = {"requests": len(reqs), "arrival_rate_hz": rate, "hbm_budget_gb": 160,
               "mix": {k: sum(1 for r in reqs if r.kind == k) for k in
                       ("quadrants2d", "blast3d_gas", "blast3d_water")},
               "cell_updates": int(sum(r.blocks * 16 ** r.dim * r.max_steps for r in reqs)),
               "step_set_cells": float(args.step_set_cells)}
        for name, prec, one, srpt in modes:
            res, mk, _ = api.serve(reqs, budget, precision=prec, one_at_a_time=one,
                                   shortest_first=srpt, step_set_cells=out["step_set_cells"])
            tts = np.array([r["finished_s"] - r["arrival_s"] for r in res])
            ok = sum(1 for r in res if r["status"] == 0)
            out[name] = {"cases_per_s": ok / mk, "makespan_s": mk,
                         "p50_tts_s": float(np.percentile(tts, 50)),
                         "p99_tts_s": float(np.percentile(tts, 99)), "completed": ok,
                         "cell_updates_per_s": out["cell_updates"] / mk}
        base = out["one_at_a_time_fp64"]
        for k, _, one, _ in modes:
            if not one:
                out[k]["cases_per_s_vs_one_at_a_time"] = out[k]["cases_per_s"] / base["cases_per_s"]
                out[k]["p50_tts_vs_one_at_a_time"] = out[k]["p50_tts_s"] / base["p50_tts_s"]
        out["bound"] = serving_bound(reqs, base["makespan_s"], fp64, engine_3d_rate)
        return out

    out = serve_stream(50.0, base_modes + srpt_modes)
    out["rates"] = {"10": serve_stream(10.0, base_modes), "200": serve_stream(200.0, base_modes)}
    return out


def water_failure_outcome(steps: int = 200):
    """The stated water configuration (spheres up to 1e9 Pa) run for `steps`
    SSP-RK3 steps in FP64 and in the FP32-flux form: where the case stops
    (ALP_ERR_NUMERIC: a cell whose stiffened-gas sound speed is not real, or a
    non-positive density) and what fails there, read from the state at the
    stop: cells with p + B <= 0 (tension beyond the stiffened-gas limit -B),
    with rho <= 0, with non-finite values."""
    import numpy as np

    from alpaca_b200 import api, cases
    from alpaca_b200 import native as N
    case = cases.water_spheres(8, seed=3, p_max=1e9, steps=steps)
    I = cases.interior(3)
    rows = []
    for prec in (N.FP64, N.FP32_FLUX):
        eng = api.Engine(3, "fvchar", precision=prec, capacity_blocks=case.grid.nb, max_cases=1)
        cid = eng.add_case(case, max_steps=steps)
        eng.run_to_end(chunk=50)
        out = np.empty_like(case.u)
        t = C.c_double()
        st = C.c_int()
        rc = N.lib().alp_engine_get_case(eng.h, cid, out.ctypes.data_as(C.POINTER(C.c_double)),
                                         C.byref(t), C.byref(st))
        eng.close()
        u = out[I]
        rho, E, m = u[:, 0], u[:, 1], u[:, 2:5]
        with np.errstate(all="ignore"):
            ke = 0.5 * (m ** 2).sum(axis=1) / rho
            p = (case.gamma - 1.0) * (E - ke) - case.gamma * case.B
        finite = np.isfinite(u).all(axis=1)
        row = {"case": "stiffened-gas water 128^3, spheres up to 1e9 Pa", "variant": "fvchar",
               "precision": "fp64" if prec == N.FP64 else "fp32-flux", "steps_asked": steps,
               "status": "ALP_ERR_NUMERIC" if rc == N.ALP_ERR_NUMERIC else
                         ("ok" if rc == N.ALP_OK else f"rc {rc}"),
               "steps_done": st.value, "t": t.value,
               "cells_p_plus_B_nonpositive": int(((p + case.B <= 0) & finite).sum()),
               "cells_rho_nonpositive": int((rho <= 0).sum()),
               "cells_nonfinite": int((~finite).sum()),
               "min_p_over_B": float(np.nanmin(np.where(finite, p, np.nan)) / case.B)}
        rows.append(row)
    return rows


def precision_report(steps: int = 200, emit=None):
    """L1 and Linf error of every field of the FP32-flux form against the FP64
    path after `steps` SSP-RK3 steps (the FP64 path is the one checked against
    the reference: per RHS <= 1e-12, 100-step L1 <= 1e-10)."""
    import numpy as np

    from alpaca_b200 import api, cases
    from alpaca_b200 import native as N
    names = ["density", "energy", "momentum_x", "momentum_y", "momentum_z"]
    rows = []
    for label, case in (("ideal gas 128^3 (512 blocks)", cases.fourier_shock(8, 3, seed=1)),
                        ("ideal gas 256^3 (4096 blocks)", cases.fourier_shock(16, 3, seed=1)),
                        ("stiffened-gas water 128^3", cases.water_spheres(8, seed=3))):
        for variant in ("fvchar", "fsroe"):
            out = {}
            failed = []
            for prec in (N.FP64, N.FP32_FLUX):
                eng = api.Engine(3, variant, precision=prec, capacity_blocks=case.grid.nb, max_cases=1)
                cid = eng.add_case(case, max_steps=steps)
                eng.run_to_end(chunk=50)
                try:
                    out[prec] = eng.get(cid)
                except N.AlpacaError as err:
                    failed.append(f"{'fp64' if prec == N.FP64 else 'fp32-flux'}: {err}")
                eng.close()
            if failed:
                row = {"case": label, "variant": variant, "failed": "; ".join(failed)}
                rows.append(row)
                if emit:
                    emit(row)
                continue
            I = cases.interior(3)
            a, b = out[N.FP32_FLUX][0][I], out[N.FP64][0][I]
            err = {}
            for f, nm in enumerate(names):
                d = np.abs(a[:, f] - b[:, f])
                err[nm] = {"l1": float(d.sum() / max(np.abs(b[:, f]).sum(), 1e-300)),
                           "linf": float(d.max() / max(np.abs(b[:, f]).max(), 1e-300))}
            row = {"case": label, "variant": variant, "steps": out[N.FP64][2],
                   "t_fp64": out[N.FP64][1], "t_fp32": out[N.FP32_FLUX][1], "errors": err}
            rows.append(row)
            if emit:
                emit(row)
    return rows


def levels_fp64_compute(args, value):
    """The face kernel bounds the multi-level step as it bounds the single-level
    one (FP64 pipe): the counted operations per cell-update against the measured
    FP64 peak (ghost fills and jump-flux kernels not counted)."""
    fp64 = fp64_peak()
    if not fp64:
        return None
    flops = FLOPS_PER_CELL_UPDATE_3D[args.variant]
    return {"flops_per_cell_update": flops, "achieved_tflops": value * flops / 1e12,
            "peak_tflops": fp64, "frac": value * flops / 1e12 / fp64,
            "peak_source": "measured FP64 FMA chains (2 flops per FMA)",
            "count": "the single-level count of the variant; ghost and jump kernels excluded"}


def levels_report(args):
    """Multi-level batching form: the 8 / 294 / 1232-leaf three-level
    spherical-shock hierarchy advanced with local time stepping (a macro step
    is 4 micro steps; level l takes 2^l RK3 steps per macro step), all levels
    in the same batched launches, one CUDA graph per macro step. Timed with
    CUDA events on the case's stream after W warm-up macro steps."""
    import torch

    from alpaca_b200 import api, cases
    case = cases.spherical_shock_levels(n0=getattr(args, "levels_n0", 4))
    prec = 1 if args.precision == "fp32" else 0
    eng = api.LevelEngine(case, args.variant, precision=prec)
    info = eng.info()
    stream = torch.cuda.ExternalStream(eng.stream_handle)
    eng.step(max(args.warmup, 3))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        e0.record(stream)
        eng.step(args.steps)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    _, t, macro = eng.get()
    eng.close()
    cu = info["cell_updates_per_macro_step"] * args.steps
    value = cu / (ms * 1e-3)
    hbm, src = peaks()
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-flux/f64-state", "data": "synthetic",
        "config": {"workload": "3d_spherical_shock_3_levels", "leaves_per_level": case.leaves_per_level(),
                   "ghost_blocks": info["ghosts"], "variant": args.variant,
                   "step": "macro step = 4 micro steps (local time stepping)",
                   "cell_updates_per_macro_step": info["cell_updates_per_macro_step"],
                   "jumps": "Multiresolution::Prediction / Average halos, "
                            "JumpFluxAdjustment conservation",
                   "sim_time_reached": t, "macro_steps_done": macro,
                   "l2": "state %.2f GB per pool > 126 MB L2 (no flush needed)"
                         % ((case.nleaf + info["ghosts"]) * 5 * 24 ** 3 * 8 / 1e9)},
        "roofline": {"bound": "hbm", "achieved": value * B_ALG_3D / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": value * B_ALG_3D / 1e9 / hbm,
                     "traffic": (LEVELS_DRAM_PER_CELL_UPDATE[(args.variant, args.precision)] *
                                 info["cell_updates_per_macro_step"]
                                 if (args.variant, args.precision) in LEVELS_DRAM_PER_CELL_UPDATE
                                 else None),
                     "traffic_note": "DRAM bytes per macro step, scaled by cell-updates from an "
                                     "ncu capture of the same hierarchy at n0 = 2",
                     "peak_source": src, "fp64_compute": levels_fp64_compute(args, value)},
        "gpu_launches": info["launches_per_macro_step"] * args.steps,
        "clocks": clocks.summary(),
    }


def run_ours(args, ws, rank, local):
    import numpy as np
    import torch

    from alpaca_b200 import api, cases
    from alpaca_b200 import native as N

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    nbd = args.blocks
    case = cases.fourier_shock(nbd, dim=3, seed=1)
    cells = case.grid.nb * 4096
    prec = N.FP32_FLUX if args.precision == "fp32" else N.FP64
    eng = api.Engine(3, args.variant, precision=prec, capacity_blocks=case.grid.nb, max_cases=1)
    stream = torch.cuda.ExternalStream(eng.stream_handle)
    cid = eng.add_case(case, max_steps=0)
    if args.path is None:
        chosen, cand_ms = eng.autotune(trial_steps=3)
    else:
        eng.set_path(args.path)
        chosen, cand_ms = args.path, None
    eng.step(args.warmup)
    torch.cuda.synchronize()
    barrier(ws, dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        e0.record(stream)
        eng.step(args.steps)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier(ws, dev)
    ms = max_over_ranks(e0.elapsed_time(e1), ws, dev)
    value = cells * args.steps * ws / (ms * 1e-3)
    u_fp64, t_sim, steps_done = eng.get(cid)
    launches = eng.launches(args.steps)
    eng.close()

    # end to end through the public C ABI from pinned host buffers: upload the
    # case's interiors, run the steps, read the interiors back (copies inside
    # the timed region; the engine keeps nothing else of a case)
    e2e = None
    if not args.no_e2e:
        inner = np.ascontiguousarray(case.u[cases.interior(3)])
        host = torch.from_numpy(inner).pin_memory()
        out = torch.empty_like(host).pin_memory()
        eng = api.Engine(3, args.variant, precision=prec, capacity_blocks=case.grid.nb,
                         max_cases=1)
        stream = torch.cuda.ExternalStream(eng.stream_handle)
        cid = eng.add_case(case, max_steps=0, interior=host.numpy())
        eng.set_path(chosen)
        eng.step(args.warmup)
        eng.remove_case(cid)
        torch.cuda.synchronize()
        barrier(ws, dev)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        cid = eng.add_case(case, max_steps=0, interior=host.numpy())
        eng.step(args.steps)
        eng.get_interior(cid, out.numpy())
        f1.record(stream)
        f1.synchronize()
        barrier(ws, dev)
        ems = max_over_ranks(f0.elapsed_time(f1), ws, dev)
        eng.close()
        nbytes = host.numel() * 8
        e2e = {"value": cells * args.steps * ws / (ems * 1e-3), "unit": METRIC,
               "h2d_bytes_per_step": nbytes / args.steps, "d2h_bytes_per_step": nbytes / args.steps,
               "ms": ems, "note": "one case per timed region: pinned H2D of the 512 blocks' "
                                  f"interiors (alp_engine_add_case_interior), {args.steps} steps, "
                                  "D2H of the final interiors (alp_engine_get_case_interior); "
                                  "bytes amortised per step"}

    # single GPU: the FP32-flux form and the multi-level batching form timed
    # beside the headline (their own lines come from --precision fp32 / --levels)
    fp32 = levels = None
    if ws == 1 and args.precision == "fp64" and not args.no_extras and args.path is None:
        eng = api.Engine(3, args.variant, precision=N.FP32_FLUX, capacity_blocks=case.grid.nb,
                         max_cases=1)
        stream = torch.cuda.ExternalStream(eng.stream_handle)
        fcid = eng.add_case(case, max_steps=0)
        f_chosen, _ = eng.autotune(trial_steps=3)
        eng.step(args.warmup)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        eng.step(args.steps)
        g1.record(stream)
        g1.synchronize()
        fms = g0.elapsed_time(g1)
        # the same case after the same W + K steps in both forms: per-field
        # relative L1 / Linf of the FP32-flux state against the FP64 one
        u_fp32, t32, s32 = eng.get(fcid)
        eng.close()
        I = cases.interior(3)
        a, b = u_fp32[I], u_fp64[I]
        errs = {}
        for f, nm in enumerate(("density", "energy", "momentum_x", "momentum_y", "momentum_z")):
            d = np.abs(a[:, f] - b[:, f])
            errs[nm] = {"l1": float(d.sum() / max(np.abs(b[:, f]).sum(), 1e-300)),
                        "linf": float(d.max() / max(np.abs(b[:, f]).max(), 1e-300))}
        fp32 = {"value": cells * args.steps / (fms * 1e-3), "unit": METRIC,
                "ms_per_step": fms / args.steps, "steps": args.steps, "warmup": args.warmup,
                "dtype": "f32-flux/f64-state", "path": CANDIDATES[f_chosen],
                "vs_fp64": ms / fms,
                "errors_vs_fp64": {"steps": s32, "same_steps": s32 == steps_done,
                                   "t_fp32": t32, "t_fp64": t_sim, "fields": errs}}
        lv = argparse.Namespace(**vars(args))
        lv.steps = min(args.steps, 20)
        lv.warmup = min(max(args.warmup, 3), 5)
        levels = levels_report(lv)
    if rank != 0:
        return
    hbm, src = peaks()
    achieved = cells * args.steps / (ms * 1e-3) * B_ALG_3D / 1e9
    fp64 = fp64_peak()
    flops = FLOPS_PER_CELL_UPDATE_3D[args.variant]
    fp64_compute = None
    if fp64:
        fp64_compute = {
            "flops_per_cell_update": flops,
            "achieved_tflops": value / ws * flops / 1e12,
            "peak_tflops": fp64, "peak_source": "measured FP64 FMA chains (2 flops per FMA)",
            "frac": value / ws * flops / 1e12 / fp64,
            "ceiling_cell_updates_per_s": fp64 * 1e12 / flops,
            "count": "add+mul+div+sqrt of the reference algorithm, counted by the oracle's "
                     "operation-counting build" + ("" if args.precision == "fp64" else
                                                   "; the FP32-flux form runs part of them in FP32")}
    cpu = None
    if not args.no_cpu_baseline:
        cpu = reference_cpu_sample(args.variant, 15.0, os.cpu_count() or 1, nblocks=args.blocks)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    clk = clocks.summary()
    serv = None
    if not args.no_serving and ws == 1:
        serv = serving_report(args, value if args.precision == "fp64" else None)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "cell_rhs_per_s": {"value": 3 * value,
                           "definition": "block right-hand sides per second, per interior cell "
                                         "(3 per SSP-RK3 cell-update, halo fills and stage "
                                         "updates included)"},
        "dtype": "f64" if args.precision == "fp64" else "f32-flux/f64-state", "data": "synthetic",
        "config": {"workload": "3d_periodic_fourier_mach2_128cubed", "blocks": case.grid.nb,
                   "cells_per_gpu": cells, "variant": args.variant,
                   "scheme": "WENO5-JS characteristic + HLLC/Einfeldt + SSP-RK3" if args.variant == "fvchar" else args.variant,
                   "cfl": 0.6, "l2": "state 283 MB per buffer > 126 MB L2 (no flush needed)",
                   "parallelism": f"replicas x{ws}", "sim_time_reached": t_sim,
                   "steps_done": steps_done,
                   "autotune": {"chosen": CANDIDATES[chosen], "candidates": CANDIDATES,
                                "ms_per_step": cand_ms}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm,
                     "traffic": TRAFFIC_PER_STEP.get((args.variant, args.precision)),
                     "peak_source": src,
                     "kernel": "whole SSP-RK3 step (one CUDA-graph launch), 320 B/cell-update",
                     "fp64_pipe_peak_tflops_measured": fp64,
                     "fp64_compute": fp64_compute},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk,
        "fp32_flux": fp32,
        "levels": levels,
        "serving": serv,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, ws, rank)
        elif args.precision_report:
            import torch
            torch.cuda.set_device(local)
            precision_report(emit=lambda row: print(json.dumps(row), flush=True))
            for row in water_failure_outcome():
                print(json.dumps(row), flush=True)
        elif args.levels:
            import torch
            torch.cuda.set_device(local)
            if rank == 0:
                print(json.dumps(levels_report(args)), flush=True)
        elif args.serving_only:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps(serving_report(args)), flush=True)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
