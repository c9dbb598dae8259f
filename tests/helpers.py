"""Shared helpers of the test suite (comparison norms, halo-filled inputs)."""
from __future__ import annotations

import numpy as np

import oracle
from alpaca_b200 import cases


def filled(case: cases.Case) -> np.ndarray:
    """The case's blocks with face halos and zero-gradient slabs filled by the oracle."""
    u = np.ascontiguousarray(case.u.copy())
    oracle.Restatement(case.grid.dim).halo_update(u, case.grid.nbr)
    return u


def field_rel_err(a: np.ndarray, b: np.ndarray, field_axis: int = 1) -> np.ndarray:
    """Per-field normwise relative error max|a-b| / max|b| (b the reference)."""
    a = np.moveaxis(a, field_axis, 0).reshape(a.shape[field_axis], -1)
    b = np.moveaxis(b, field_axis, 0).reshape(b.shape[field_axis], -1)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return np.abs(a - b).max(axis=1) / scale


def field_rel_err_floored(a: np.ndarray, b: np.ndarray, field_axis: int = 1) -> np.ndarray:
    """field_rel_err, except that a field whose reference is identically zero
    (e.g. the mass right-hand side of a scheme without dissipation on a fluid
    at rest) is measured against the largest field's scale."""
    a2 = np.moveaxis(a, field_axis, 0).reshape(a.shape[field_axis], -1)
    b2 = np.moveaxis(b, field_axis, 0).reshape(b.shape[field_axis], -1)
    scale = np.abs(b2).max(axis=1)
    scale = np.where(scale > 0.0, scale, max(scale.max(), 1e-300))
    return np.abs(a2 - b2).max(axis=1) / scale


def l1_rel(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


def small_cases():
    """Small seeded cases in 1, 2 and 3 dimensions (seconds on the CPU oracle)."""
    return {
        1: cases.sod_1d(),
        2: cases.fourier_shock(2, dim=2, seed=3),
        3: cases.fourier_shock(1, dim=3, seed=5),
    }
