"""Seeded request streams of the serving form: independent 2D four-quadrant
Riemann problems and 3D spherical blasts (ideal gas or stiffened-gas water),
log-uniform sizes of 4 to 2048 blocks of 16^d cells, 200-2000 SSP-RK3 steps
each, Poisson arrivals. Water is non-dimensionalised as the reference's
UnitHandler does (unit_handler.cpp:33-56) with rho_ref = 1000 kg/m^3,
u_ref = sqrt(p_ref / rho_ref), p_ref = 1e5 Pa, L_ref = 1 m."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import native as N

WATER_GAMMA = 6.12
WATER_B_PA = 3.43e8


class UnitHandler:
    """Reference quantities of unit_handler.cpp:33-56."""

    def __init__(self, density, velocity, length, temperature=1.0):
        self.density = density
        self.velocity = velocity
        self.length = length
        self.temperature = temperature
        self.time = length / velocity
        self.pressure = density * velocity * velocity
        self.energy = density * velocity * velocity
        self.momentum = density * velocity

    def nd(self, value, kind: str):
        return value / getattr(self, kind)


WATER_UNITS = UnitHandler(1000.0, math.sqrt(1e5 / 1000.0), 1.0)


@dataclass
class Request:
    dim: int
    nblocks: tuple
    cell_size: float
    gamma: float
    B: float
    ic_type: int
    params: list
    max_steps: int
    arrival_s: float = 0.0
    cfl: float = 0.6
    t_end: float = 1e300
    periodic: tuple = (0, 0, 0)
    kind: str = field(default="")
    program: object = None  # api.IcProgram for ic_type IC_PROGRAM
    origin: tuple = (0.0, 0.0, 0.0)
    units: tuple | None = None  # (density, velocity, length) references

    @property
    def blocks(self) -> int:
        return self.nblocks[0] * self.nblocks[1] * self.nblocks[2]


def grid_shape(nb_target: int, dim: int):
    """Near-square / near-cubic block grid with about nb_target blocks."""
    side = max(1, round(nb_target ** (1.0 / dim)))
    shape = [side] * dim
    # adjust the first dimension to approach the target
    rest = int(np.prod(shape[1:])) if dim > 1 else 1
    shape[0] = max(1, round(nb_target / rest))
    return tuple(shape) + (1,) * (3 - dim)


def quadrant_request(rng, nb_target: int, steps: int) -> Request:
    """2D four-quadrant Riemann problem: per quadrant rho, p ~ U(0.1, 2),
    u, v ~ U(-1, 1), ideal gas gamma 1.4, on the unit square's largest side."""
    shape = grid_shape(nb_target, 2)
    h = 1.0 / (16 * max(shape[:2]))
    params = [0.5 * shape[0] * 16 * h, 0.5 * shape[1] * 16 * h]
    for _ in range(4):
        rho, p = rng.uniform(0.1, 2.0, 2)
        u, v = rng.uniform(-1.0, 1.0, 2)
        params += [rho, u, v, p]
    return Request(2, shape, h, 1.4, 0.0, N.IC_QUADRANTS, params, steps, kind="quadrants2d")


def blast_request(rng, nb_target: int, steps: int, water: bool) -> Request:
    """3D spherical blast at the box centre, radius 0.2 of the largest side,
    pressure ratio U(10, 1000); ideal gas (rho 1, p 1 outside) or stiffened-gas
    water (1000 kg/m^3, 1e5 Pa outside, gamma 6.12, B 3.43e8 Pa)."""
    shape = grid_shape(nb_target, 3)
    h = 1.0 / (16 * max(shape))
    ratio = rng.uniform(10.0, 1000.0)
    centre = [0.5 * n * 16 * h for n in shape]
    if water:
        gamma, B = WATER_GAMMA, WATER_UNITS.nd(WATER_B_PA, "pressure")
        rho, p_out = WATER_UNITS.nd(1000.0, "density"), WATER_UNITS.nd(1e5, "pressure")
    else:
        gamma, B, rho, p_out = 1.4, 0.0, 1.0, 1.0
    params = centre + [0.2, rho, p_out * ratio, rho, p_out]
    return Request(3, shape, h, gamma, B, N.IC_BLAST, params, steps,
                   kind="blast3d_water" if water else "blast3d_gas")


def request_stream(n: int, seed: int = 0, rate_hz: float = 50.0, min_blocks: int = 4,
                   max_blocks: int = 2048, min_steps: int = 200, max_steps: int = 2000,
                   frac_2d: float = 0.5, frac_water: float = 0.5):
    """n requests with Poisson arrivals at rate_hz, log-uniform block counts and
    uniform step budgets."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += rng.exponential(1.0 / rate_hz)
        nb = int(round(math.exp(rng.uniform(math.log(min_blocks), math.log(max_blocks)))))
        steps = int(rng.integers(min_steps, max_steps + 1))
        if rng.uniform() < frac_2d:
            r = quadrant_request(rng, nb, steps)
        else:
            r = blast_request(rng, nb, steps, water=rng.uniform() < frac_water)
        r.arrival_s = t
        out.append(r)
    return out
