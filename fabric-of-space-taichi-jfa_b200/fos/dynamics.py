"""Drop-in for the hot-path kernels of the reference's dynamics.py on libfos.

Same names and argument order as dynamics.py (cited per function); tensors in
place of Taichi fields.  apply_brownian_motion draws its jitter from
Philox-4x32-10 keyed by the configured seed and a per-call counter, in place
of ti.random().
"""
from __future__ import annotations

from . import runtime

_brownian_calls = 0
_jitter_calls = 0


def _t(x):
    return getattr(x, "tensor", x)


def project_overlaps(pos, rad, cell_start, cell_count, cell_indices, n: int):
    """dynamics.project_overlaps (dynamics.py:77-171), one Jacobi sweep."""
    runtime.ctx().project_overlaps(_t(pos), _t(rad), _t(cell_start), _t(cell_count),
                                   _t(cell_indices), n)


def compute_max_overlap(pos, rad, cell_start, cell_count, cell_indices, local_max_depth,
                        n: int) -> float:
    """dynamics.compute_max_overlap (dynamics.py:367-372)."""
    return runtime.ctx().compute_max_overlap(_t(pos), _t(rad), _t(cell_start), _t(cell_count),
                                             _t(cell_indices), _t(local_max_depth), n)


def equilibrate_pressure(n, frame, pos, rad, delta_r, jfa_face_ids, jfa_fsc, k, P_exp,
                         pair_cap, max_nei, r_min, r_max):
    """dynamics.equilibrate_pressure (dynamics.py:1454-1557) -> (max|dr|, changed)."""
    return runtime.ctx().equilibrate_pressure(int(n), int(frame), _t(rad), _t(delta_r),
                                              _t(jfa_face_ids), _t(jfa_fsc), k, P_exp, pair_cap,
                                              max_nei, r_min, r_max, sweeps=1)


def set_fsc_targets(rad, rad_target, fsc, fsc_ema, n, f_low, f_high, growth_pct, r_min, r_max):
    """dynamics.set_fsc_targets (dynamics.py:1242-1320)."""
    runtime.ctx().set_fsc_targets(_t(rad), _t(rad_target), _t(fsc), _t(fsc_ema), n, f_low, f_high,
                                  growth_pct, r_min, r_max)


def nudge_radii_adaptive_ema(rad, rad_target, local_max_depth, n, alpha, max_step_pct, r_min,
                             r_max, back_global, mode):
    """dynamics.nudge_radii_adaptive_ema (dynamics.py:1366-1427)."""
    runtime.ctx().nudge_radii(_t(rad), _t(rad_target), _t(local_max_depth), n, alpha,
                              max_step_pct, r_min, r_max, back_global, mode)


def compute_controller_stats(rad, rad_target, fsc_ema, n, f_low, f_high):
    """dynamics.compute_controller_stats (dynamics.py:1322-1363)."""
    return runtime.ctx().controller_stats(_t(rad), _t(rad_target), _t(fsc_ema), n, f_low, f_high)


def compute_pressure_stats(n, rad, P_exp, r_min, r_max):
    """dynamics.compute_pressure_stats (dynamics.py:1560-1589) -> (rmin, rmax)."""
    return runtime.ctx().pressure_stats(n, _t(rad))


def apply_brownian_motion(pos, n, strength, domain_size):
    """dynamics.apply_brownian_motion (dynamics.py:1596-1634)."""
    global _brownian_calls
    runtime.ctx().apply_brownian(_t(pos), n, strength, domain_size, runtime.config().SEED,
                                 _brownian_calls)
    _brownian_calls += 1


def init_jitter_velocities(v_jit, n: int):
    """dynamics.init_jitter_velocities (dynamics.py:600-605)."""
    runtime.ctx().init_jitter_velocities(_t(v_jit), n)


def compute_mean_radius(rad, n: int, mean_radius):
    """dynamics.compute_mean_radius (dynamics.py:675-689) into the one-element
    float32 tensor mean_radius (exact sum, rounded once)."""
    runtime.ctx().compute_mean_radius(_t(rad), n, _t(mean_radius))


def apply_brownian(v_jit, rad, mean_radius, n: int, dt: float):
    """dynamics.apply_brownian (dynamics.py:607-646): OU update of v_jit with
    JITTER_RMS / JITTER_TAU / MAX_DRIFT_FRACTION / GAP_FRACTION of the
    configuration; the draws are Philox-4x32-10 keyed by the configured seed
    and a per-call counter."""
    global _jitter_calls
    cfg = runtime.config()
    runtime.ctx().apply_jitter(_t(v_jit), _t(rad), _t(mean_radius), n, dt, cfg.JITTER_RMS,
                               cfg.JITTER_TAU, cfg.MAX_DRIFT_FRACTION, cfg.GAP_FRACTION,
                               cfg.SEED, _jitter_calls)
    _jitter_calls += 1


def integrate_jitter(pos, v_jit, n: int, dt: float):
    """dynamics.integrate_jitter (dynamics.py:649-660): pos = wrapP(pos + v dt)."""
    runtime.ctx().integrate_jitter(_t(pos), _t(v_jit), n, dt)


def alpha_for_frames(frames: int) -> float:
    """run.py:440-452"""
    return 1.0 - (0.05 ** (1.0 / max(1, frames)))


def backpressure_from_overlap(o_max: float, contact_tol: float) -> float:
    """run.py:454-470"""
    if contact_tol <= 0:
        return 1.0
    raw = (contact_tol - o_max) / contact_tol
    return max(0.25, min(1.0, raw))
