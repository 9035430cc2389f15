"""Shared helpers for the parity tests: workloads and oracle/GPU parameter sets."""
from __future__ import annotations

import numpy as np

from fos import inputs
from oracle import oracle as O


def wrapped(pos: np.ndarray, L: float = 1.0) -> np.ndarray:
    """grid.wrapP (grid.py:30-48) in float32, as initialize_simulation applies it."""
    f = np.float32
    p = np.ascontiguousarray(pos, np.float32).copy()
    return p - f(L) * np.floor(p * f(1.0 / L) + f(0.5))


def oracle_params(foam, **over) -> O.OracleParams:
    kw = dict(n=foam.n, L=1.0, R=foam.res, r_max_cell=foam.r_max, f_low=foam.f_low,
              f_high=foam.f_high, r_min=foam.r_min, r_max=foam.r_max, brownian=1e-4,
              seed=foam.seed, pbd_iters=foam.pbd_iters, pressure_iters=foam.pressure_iters,
              jfa_warm=foam.jfa_warm, jfa_cadence=foam.jfa_cadence)
    kw.update(over)
    return O.OracleParams(**kw)


def foam(name: str):
    return {"small": inputs.small, "headline": inputs.headline, "stress": inputs.stress}[name]()
