"""Seeded synthetic foams for the five benchmark workloads.

The reference seeds its foam in run.py:239-291 (np.random.uniform positions in
the centred box, radii R_START*(1 +- 0.3 U) clipped).  The workloads below keep
that structure -- positions first, then radii, float32 -- with the sizes and
radius laws of the five named workloads.  Generator: numpy PCG64 via
``np.random.default_rng(seed)``.  Positions are drawn in the unit cube [0,1)^3
and wrapped into [-L/2, L/2)^3 by grid.wrapP (grid.py:30-48) before first use.

Each workload also fixes the controller's radius bounds (R_MIN/R_MAX), which
the reference takes from config.py:49-50 for its own box; here they are the
radius law's clip range so the hash-grid cell of 2*r_max stays valid.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Foam:
    name: str
    pos: np.ndarray          # [N,3] float32 in [0,1)^3 (unwrapped)
    rad: np.ndarray          # [N] float32
    res: int                 # JFA_RES
    r_min: float             # controller lower bound
    r_max: float             # controller upper bound; hash cell = 2*r_max
    f_low: int
    f_high: int
    pbd_iters: int
    pressure_iters: int
    jfa_warm: int            # frames with JFA every frame
    jfa_cadence: int         # then JFA every k-th frame
    frames: int
    seed: int

    @property
    def n(self) -> int:
        return int(self.rad.shape[0])


def _uniform_pos(rng, n):
    return rng.random((n, 3), dtype=np.float32)


def small(seed: int = 0) -> Foam:
    """N=1,000, r ~ U[0.025, 0.035], 64^3, JFA every frame, band [10,16], K=4, M=10."""
    rng = np.random.default_rng(seed)
    pos = _uniform_pos(rng, 1000)
    rad = rng.uniform(0.025, 0.035, 1000).astype(np.float32)
    return Foam("small-1k-64", pos, rad, 64, 0.0125, 0.035, 10, 16, 4, 10, 1 << 30, 1, 100, seed)


def headline(seed: int = 1) -> Foam:
    """N=10,000, lognormal r (median 0.015, sigma_log 0.25) clipped to [0.007, 0.03],
    128^3, 20 warm-start frames with JFA every frame then every 5th, K=8, M=20, band [12,16]."""
    rng = np.random.default_rng(seed)
    pos = _uniform_pos(rng, 10000)
    rad = np.clip(rng.lognormal(np.log(0.015), 0.25, 10000), 0.007, 0.03).astype(np.float32)
    return Foam("headline-10k-128", pos, rad, 128, 0.007, 0.03, 12, 16, 8, 20, 20, 5, 1000, seed)


def stress(seed: int = 2) -> Foam:
    """N=200,000, bimodal r: 50% U[0.004,0.005], 50% U[0.007,0.009], 256^3, JFA every frame."""
    rng = np.random.default_rng(seed)
    n = 200000
    pos = _uniform_pos(rng, n)
    small_mode = rng.random(n) < 0.5
    r = np.where(small_mode, rng.uniform(0.004, 0.005, n), rng.uniform(0.007, 0.009, n))
    return Foam("stress-200k-256", pos, r.astype(np.float32), 256, 0.002, 0.009, 12, 16, 8, 20,
                1 << 30, 1, 200, seed)


def surrogate_variant(seed: int = 10, large: bool = False) -> Foam:
    """Foams of the FSC surrogate: the headline workload's law (training uses
    seeds 10-19), or the 50,000-particle variant whose radii follow the same
    law scaled by (1/5)^(1/3), on a 192^3 grid."""
    if not large:
        return headline(seed)
    rng = np.random.default_rng(seed)
    n = 50000
    s = (1.0 / 5.0) ** (1.0 / 3.0)
    pos = _uniform_pos(rng, n)
    rad = (np.clip(rng.lognormal(np.log(0.015), 0.25, n), 0.007, 0.03) * s).astype(np.float32)
    return Foam("surrogate-50k-192", pos, rad, 192, 0.007 * s, 0.03 * s, 12, 16, 8, 20, 20, 5,
                1000, seed)


ENSEMBLE_RES = (64, 96, 128)


def ensemble_member(n: int, seed: int, band_low: int = 12, name: str = "ensemble") -> Foam:
    """One foam of the batched ensemble: uniform positions, lognormal radii with
    median 0.03*(1000/N)^(1/3) and sigma_log 0.25 (clipped to [0.4, 2] x median),
    JFA_RES the smallest of 64/96/128 with R^3/N >= 100, band [low, low + 4],
    K=8 PBD and M=20 pressure sweeps, 20 warm-start frames then JFA every 5th."""
    rng = np.random.default_rng(seed)
    med = 0.03 * (1000.0 / n) ** (1.0 / 3.0)
    pos = _uniform_pos(rng, n)
    rad = rng.lognormal(np.log(med), 0.25, n)
    lo_clip, hi_clip = 0.4 * med, 2.0 * med
    rad = np.clip(rad, lo_clip, hi_clip).astype(np.float32)
    res = next((r for r in ENSEMBLE_RES if r ** 3 / n >= 100), ENSEMBLE_RES[-1])
    return Foam(name, pos, rad, res, lo_clip, hi_clip, band_low, band_low + 4, 8, 20, 20, 5, 500,
                seed)


def ensemble(seed: int = 3, count: int = 64, n_range=(2000, 20000)) -> list[Foam]:
    """The batched-ensemble workload: `count` independent foams with N drawn
    uniformly from n_range (seed 3), per-foam band low ~ U{10..14}; each foam
    is ensemble_member(N, seed * 1000 + k, low)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        low = int(rng.integers(10, 15))
        out.append(ensemble_member(n, seed * 1000 + k, low, name=f"ensemble-{k}"))
    return out


WORKLOADS = {"small": small, "headline": headline, "stress": stress}
