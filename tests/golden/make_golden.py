"""Generates the golden fixtures of tests/golden/ from the reference itself.

The outputs come from tumaer/ALPACA's own hot-path sources, compiled in place
by oracle/Makefile into oracle/_ref/ (run `make -C oracle ref` first, with the
reference sources available). Inputs are the seeded workloads of
alpaca_b200/cases.py; each fixture stores the sha256 of its input so a test can
tell that the generator still reproduces it bit for bit.

    python tests/golden/make_golden.py            # small fixtures
    python tests/golden/make_golden.py --c2       # also the 128^3, 100-step run summary
    python tests/golden/make_golden.py --ext      # the further selections (make -C oracle ref-ext)
    python tests/golden/make_golden.py --ext fs_weno3   # only the named selections
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from alpaca_b200 import cases  # noqa: E402
from helpers import filled, small_cases  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def rhs_fixtures():
    for dim, case in small_cases().items():
        u = filled(case)
        I = cases.interior(dim)
        for variant in oracle.VARIANTS:
            ref = oracle.Reference(dim, variant)
            fx, fy, fz, rhs = ref.space_rhs(u, case.gamma, case.B, False, case.grid.cell_size)
            dt = oracle.Restatement(dim).timestep(u, case.gamma, case.B, False,
                                                  case.grid.cell_size, case.cfl)
            path = os.path.join(HERE, f"rhs_d{dim}_{variant}.npz")
            np.savez_compressed(path, input_sha=sha(u), rhs=rhs[I], dt=dt,
                                case=case.name, cell_size=case.grid.cell_size)
            print("wrote", path)


def sod_fixtures():
    case = cases.sod_1d()
    I = cases.interior(1)
    for variant in oracle.VARIANTS:
        ref = oracle.Reference(1, variant)
        u, t, steps, dts = ref.run(case.u, case.grid.nbr, case.gamma, case.B, False,
                                   case.grid.cell_size, case.cfl, case.t_end)
        path = os.path.join(HERE, f"sod1d_{variant}.npz")
        np.savez_compressed(path, input_sha=sha(case.u), final=u[I], t=t, steps=steps, dts=dts)
        print("wrote", path, steps, t)


def short_run_fixtures(nsteps: int = 5):
    for dim in (2, 3):
        case = small_cases()[dim]
        I = cases.interior(dim)
        for variant in oracle.VARIANTS:
            ref = oracle.Reference(dim, variant)
            u, t, steps, dts = ref.run(case.u, case.grid.nbr, case.gamma, case.B, False,
                                       case.grid.cell_size, case.cfl, 1e300, max_steps=nsteps,
                                       nthreads=os.cpu_count() or 1)
            path = os.path.join(HERE, f"run{nsteps}_d{dim}_{variant}.npz")
            np.savez_compressed(path, input_sha=sha(case.u), final=u[I], t=t, steps=steps,
                                dts=dts)
            print("wrote", path)


def ext_fixtures(only=()):
    """1D and 3D right-hand sides and the 1D Sod run of every further selection
    (stencils, Riemann solvers, signal speeds, flux splittings), or of the
    named ones."""
    for variant in only or oracle.EXT_VARIANTS:
        for dim in (1, 3):
            case = small_cases()[dim]
            u = filled(case)
            I = cases.interior(dim)
            rhs = oracle.Reference(dim, variant).space_rhs(u, case.gamma, case.B, False,
                                                           case.grid.cell_size)[3]
            path = os.path.join(HERE, "ext", f"rhs_d{dim}_{variant}.npz")
            np.savez_compressed(path, input_sha=sha(u), rhs=rhs[I])
        case = cases.sod_1d()
        u, t, steps, dts = oracle.Reference(1, variant).run(
            case.u, case.grid.nbr, case.gamma, case.B, False, case.grid.cell_size, case.cfl,
            case.t_end)
        path = os.path.join(HERE, "ext", f"sod1d_{variant}.npz")
        np.savez_compressed(path, input_sha=sha(case.u), final=u[cases.interior(1)], t=t,
                            steps=steps, dts=dts)
        print("wrote", variant, steps, t)


def c2_summary(variant: str, steps: int = 100):
    """The 3D periodic 128^3 Fourier + Mach-2 shock case after `steps` RK3 steps:
    per-block per-field interior sums and every 8th cell, from the reference."""
    case = cases.fourier_shock(8, dim=3, seed=1, steps=steps)
    ref = oracle.Reference(3, variant)
    t0 = time.time()
    u, t, n, dts = ref.run(case.u, case.grid.nbr, case.gamma, case.B, False,
                           case.grid.cell_size, case.cfl, 1e300, max_steps=steps,
                           nthreads=os.cpu_count() or 1)
    I = cases.interior(3)
    glob = case.grid.gather(u)
    path = os.path.join(HERE, f"c2_128_{variant}_{steps}steps.npz")
    np.savez_compressed(path, input_sha=sha(case.u), block_sums=u[I].sum(axis=(2, 3, 4)),
                        sub=glob[:, ::8, ::8, ::8], t=t, steps=n, dts=dts,
                        seconds=time.time() - t0, threads=os.cpu_count() or 1)
    print("wrote", path, n, t, f"{time.time() - t0:.0f}s")


if __name__ == "__main__":
    if not oracle.Reference.available():
        sys.exit("oracle/_ref is not built: run `make -C oracle ref` with the reference sources")
    if "--ext" in sys.argv:
        os.makedirs(os.path.join(HERE, "ext"), exist_ok=True)
        # --ext [name ...]: all further selections, or only the named ones
        ext_fixtures(tuple(a for a in sys.argv[sys.argv.index("--ext") + 1:]
                           if not a.startswith("--")))
        sys.exit(0)
    rhs_fixtures()
    sod_fixtures()
    short_run_fixtures()
    if "--c2" in sys.argv:
        for v in ("fvchar", "fsroe"):
            c2_summary(v)
