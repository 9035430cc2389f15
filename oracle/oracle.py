"""ctypes front end and frame driver for the CPU restatement (fos_oracle.c).

TEST INFRASTRUCTURE ONLY: the parity checker and the CPU baseline.  Nothing in
the product package imports this module; only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg do.

Parity against the reference itself is UNPINNED (the reference is Taichi code,
Taichi is not installable here, and the reference has no golden vectors); the
restatement is pinned by the analytic known-answer tests in
tests/test_oracle_kat.py.

Every function cites the reference file:line it restates.  Constants that
Taichi folds from Python globals are folded here in double precision and
rounded to float32 once (``_f32``), which is what Taichi does when it bakes a
Python float into a kernel as an f32 literal.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

S = 32  # MAX_NEIGHBORS (jfa.py:74)

_f = C.c_float
_i = C.c_int
_p = C.c_void_p


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "orc_jfa_init": (None, [_p, _p, _i, _i, _f, _f, _f, _f, _p]),
            "orc_jfa_pass": (C.c_longlong, [_p, _p, _p, _p, _i, _f, _f, _f, _f, _i, _i]),
            "orc_jfa_run": (_i, [_p, _p, _i, _i, _f, _f, _f, _f, _i, _i, _i, C.c_double, _i,
                                 _p, _p, _p]),
            "orc_majority_filter": (None, [_p, _i, _p]),
            "orc_accumulate_faces": (None, [_p, _i, _i, _p, _p]),
            "orc_finalize": (None, [_i, _p, _p, _p, _f, _f, _f, _f, _p, _p, _p, _p]),
            "orc_fsc_ema": (None, [_i, _p, _p, _f]),
            "orc_grid_build": (None, [_p, _i, _i, _f, _f, _f, _p, _p, _p]),
            "orc_pbd": (None, [_p, _p, _p, _i, _i, _f, _f, _f, _p, _p, _p, _f, _f, _f]),
            "orc_max_overlap": (_f, [_p, _p, _i, _i, _f, _f, _f, _p, _p, _p, _f, _p]),
            "orc_pressure": (_f, [_i, _i, _p, _p, _p, _p, _f, _f, _f, _i, _f, _f, _p]),
            "orc_philox": (None, [C.c_uint32] * 6 + [_p]),
            "orc_brownian": (None, [_p, _i, _f, _f, C.c_uint64, C.c_uint32]),
            "orc_mean_radius": (_f, [_p, _i]),
            "orc_dirty_mark": (None, [_p, _p, _p, _p, _i, _i, _f, _f, _f, _f, _i, _p]),
            "orc_dirty_count": (_i, [_p, _i]),
            "orc_topo_candidates": (None, [_p, _p, _p, _p, _p, _i, _i, _f, _f, _f, _f, _i, _p,
                                           _p, _p]),
            "orc_topo_gabriel": (None, [_p, _p, _p, _p, _i, _i, _f, _f, _f, _f, _i, _i, _i,
                                        _f, _i, _p, _p, _p, _p]),
            "orc_topo_batched": (None, [_p, _p, _p, _p, _p, _i, _i, _f, _f, _f, _f, _f, _i, _i,
                                        _i, _i, _i, _p, _p, _p, _p]),
            "orc_topo_knn": (None, [_p, _p, _p, _p, _p, _i, _i, _f, _f, _f, _f, _i, _p]),
            "orc_topo_ema": (None, [_p, _p, _f, _i]),
            "orc_topo_radii": (None, [_p, _p, _f, _f, _f, _f, _f, _f, _i]),
            "orc_ou_jitter": (None, [_p, _p, _p, _i, _f, _f, C.c_double, C.c_double, C.c_double,
                                     C.c_double, _f, _f, C.c_uint64, C.c_uint32]),
            "orc_set_targets": (None, [_p, _p, _p, _p, _i, _i, _i, _f, _f, _f, _f]),
            "orc_nudge": (None, [_p, _p, _p, _i, _f, _f, _f, _f, _f, _i, _f]),
            "orc_num_threads": (_i, []),
            "orc_set_threads": (None, [_i]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def _f32(x: float) -> float:
    return float(np.float32(x))


# --------------------------------------------------------------------- params
@dataclass
class OracleParams:
    """Constants of config.py / jfa.py, overridable per workload."""
    n: int
    L: float = 1.0                    # DOMAIN_SIZE
    R: int = 128                      # JFA_RES
    r_max_cell: float = 0.03          # cell size = 2 * r_max_cell
    beta: float = 1.0                 # POWER_BETA (jfa.py:184)
    early_exit: bool = False          # JFA_EARLY_EXIT_ENABLED (config.py:208)
    min_passes: int = 3               # MIN_JFA_PASSES
    th_delta: float = 0.006           # TH_PASS_DELTA
    tie_lower: bool = False
    face_scale: float = 1.5           # EXPECTED_FACE_SCALE (jfa.py:58)
    t_add: float = 0.15               # T_ADD (jfa.py:63)
    t_drop: float = 0.10              # T_DROP (jfa.py:64)
    ema_alpha: float = 0.33           # JFA_EMA_ALPHA (config.py:81)
    gap: float = 0.015                # GAP_FRACTION
    mdf: float = 0.2                  # MAX_DISPLACEMENT_FRAC
    dmul: float = 2.0                 # DISPLACEMENT_MULTIPLIER
    eps: float = 1e-8                 # EPS
    contact_tol: float = 0.035        # CONTACT_TOL
    k: float = 0.10                   # PRESSURE_K
    P: float = 3.0                    # PRESSURE_EXP
    pair_cap: float = 0.02            # PRESSURE_PAIR_CAP
    max_nei: int = 10                 # MAX_EQ_NEI
    f_low: int = 12
    f_high: int = 16
    growth: float = 0.10              # GROWTH_PCT
    max_step: float = 0.12            # MAX_STEP_PCT
    adjust_frames: int = 15           # ADJUSTMENT_FRAMES
    deadband: float = 1.0             # FSC_DEADBAND
    bp_mode: int = 2                  # BACKPRESSURE_MODE "local"
    warm_frames: int = 30             # WARMSTART_FRAMES (growth gate)
    zero_thresh: float = 0.10         # FSC_ZERO_RATE_THRESH
    r_min: float = 0.007
    r_max: float = 0.03
    brownian: float = 1e-4
    seed: int = 1
    pbd_iters: int = 8
    pressure_iters: int = 20
    jfa_warm: int = 20
    jfa_cadence: int = 5
    warmup_pbd: int = 4               # PBD_BASE_PASSES
    ou: bool = False                  # JITTER_ENABLED (config.py:493; off for the workloads)
    jitter_rms: float = 0.10          # JITTER_RMS
    jitter_tau: float = 1.0           # JITTER_TAU
    dt: float = 0.016                 # DT
    max_drift: float = 0.20           # MAX_DRIFT_FRACTION

    @property
    def G(self) -> int:
        # GRID_RES = max(3, ceil(L / CELL_SIZE)) (config.py:317)
        return max(3, int(math.ceil(self.L / (2.0 * self.r_max_cell))))

    @property
    def passes(self) -> int:
        # JFA_NUM_PASSES = ceil(log2 R) + 1 (jfa.py:223)
        return int(np.ceil(np.log2(self.R))) + 1

    @property
    def vs(self) -> float:
        return _f32(self.L / self.R)  # VOXEL_SIZE (jfa.py:220)

    @property
    def halfL(self) -> float:
        return _f32(0.5 * self.L)

    @property
    def invL(self) -> float:
        return _f32(1.0 / self.L)  # INV_L (config.py:214)

    def is_jfa_frame(self, f: int) -> bool:
        return f < self.jfa_warm or f % self.jfa_cadence == 0


# ------------------------------------------------------------- stage wrappers
def jfa_init(pos, rad, p: OracleParams):
    lab = np.empty(p.R ** 3, np.int32)
    lib().orc_jfa_init(_ptr(pos), _ptr(rad), p.n, p.R, _f32(p.L), p.halfL, p.vs, _f32(p.beta),
                       _ptr(lab))
    return lab


def jfa_pass(lab_in, pos, rad, p: OracleParams, step: int):
    out = np.empty_like(lab_in)
    ch = lib().orc_jfa_pass(_ptr(lab_in), _ptr(out), _ptr(pos), _ptr(rad), p.R, _f32(p.L),
                            p.halfL, p.vs, _f32(p.beta), step, int(p.tie_lower))
    return out, int(ch)


def jfa_labels(pos, rad, p: OracleParams):
    """jfa_init + pass loop (jfa.py:1075-1116). Returns (labels, changes, passes)."""
    lab = np.empty(p.R ** 3, np.int32)
    scr = np.empty(p.R ** 3, np.int32)
    ch = np.zeros(64, np.int64)
    done = lib().orc_jfa_run(_ptr(pos), _ptr(rad), p.n, p.R, _f32(p.L), p.halfL, p.vs,
                             _f32(p.beta), p.passes, int(p.early_exit), p.min_passes,
                             float(p.th_delta), int(p.tie_lower), _ptr(lab), _ptr(scr), _ptr(ch))
    return lab, ch[:done].copy(), int(done)


def majority_filter(lab, R):
    out = np.empty_like(lab)
    lib().orc_majority_filter(_ptr(lab), R, _ptr(out))
    return out


def accumulate_faces(filt, R, n):
    ids = np.empty((n, S), np.int32)
    cnt = np.empty((n, S), np.int32)
    lib().orc_accumulate_faces(_ptr(filt), R, n, _ptr(ids), _ptr(cnt))
    return ids, cnt


def finalize(rad, ids, cnt, prev, p: OracleParams):
    """finalize_faces_kernel (jfa.py:788-857); prev is updated in place."""
    n = p.n
    nl = np.empty((n, S), np.int32)
    used = np.empty(n, np.int32)
    fsc = np.empty(n, np.int32)
    lib().orc_finalize(n, _ptr(rad), _ptr(ids), _ptr(cnt), p.vs, _f32(p.face_scale),
                       _f32(p.t_add), _f32(p.t_drop), _ptr(prev), _ptr(nl), _ptr(used), _ptr(fsc))
    return nl, used, fsc


def fsc_ema(fsc, ema, alpha):
    lib().orc_fsc_ema(len(fsc), _ptr(fsc), _ptr(ema), _f32(alpha))


def grid_build(pos, p: OracleParams):
    G = p.G
    cc = np.empty(G ** 3, np.int32)
    cs = np.empty(G ** 3, np.int32)
    ci = np.empty(p.n, np.int32)
    lib().orc_grid_build(_ptr(pos), p.n, G, _f32(p.L), p.invL, p.halfL, _ptr(cc), _ptr(cs),
                         _ptr(ci))
    return cc, cs, ci


def pbd(pos, rad, grid, p: OracleParams):
    cc, cs, ci = grid
    out = np.empty_like(pos)
    lib().orc_pbd(_ptr(pos), _ptr(out), _ptr(rad), p.n, p.G, _f32(p.L), p.invL, p.halfL,
                  _ptr(cs), _ptr(cc), _ptr(ci), _f32(1.0 + p.gap), _f32(p.mdf), _f32(p.dmul))
    return out


def max_overlap(pos, rad, grid, p: OracleParams):
    cc, cs, ci = grid
    lm = np.empty(p.n, np.float32)
    g = lib().orc_max_overlap(_ptr(pos), _ptr(rad), p.n, p.G, _f32(p.L), p.invL, p.halfL,
                              _ptr(cs), _ptr(cc), _ptr(ci), _f32(p.eps), _ptr(lm))
    return float(g), lm


def pressure(rad, ids, fsc, frame, p: OracleParams):
    dr = np.empty(p.n, np.float32)
    ch = C.c_int(0)
    mx = lib().orc_pressure(p.n, int(frame), _ptr(rad), _ptr(dr), _ptr(ids), _ptr(fsc),
                            _f32(p.k), _f32(p.P), _f32(p.pair_cap), p.max_nei, _f32(p.r_min),
                            _f32(p.r_max), C.byref(ch))
    return float(mx), int(ch.value), dr


def philox(ctr, key):
    out = np.empty(4, np.uint32)
    lib().orc_philox(*(int(c) & 0xFFFFFFFF for c in ctr), *(int(k) & 0xFFFFFFFF for k in key),
                     _ptr(out))
    return out


def brownian(pos, p: OracleParams, frame: int):
    lib().orc_brownian(_ptr(pos), p.n, _f32(p.brownian), _f32(p.L), int(p.seed), int(frame))


def mean_radius(rad, n: int) -> float:
    return float(lib().orc_mean_radius(_ptr(rad), int(n)))


def ou_jitter(pos, v_jit, rad, p: OracleParams, frame: int):
    """Frame step 6B (run.py:855-867): mean radius, apply_brownian,
    integrate_jitter."""
    m = mean_radius(rad, p.n)
    lib().orc_ou_jitter(_ptr(pos), _ptr(v_jit), _ptr(rad), p.n, _f32(m), _f32(p.dt),
                        float(p.jitter_rms), float(p.jitter_tau), float(p.max_drift),
                        float(p.gap), _f32(p.L), p.invL, int(p.seed),
                        int(frame))


def set_targets(rad, rad_target, fsc, ema, p: OracleParams):
    lib().orc_set_targets(_ptr(rad), _ptr(rad_target), _ptr(fsc), _ptr(ema), p.n, p.f_low,
                          p.f_high, _f32(p.growth), _f32(p.r_min), _f32(p.r_max),
                          _f32(p.deadband))


def alpha_for_frames(frames: int) -> float:
    """run.py:440-452"""
    return 1.0 - (0.05 ** (1.0 / max(1, frames)))


def backpressure_from_overlap(o_max: float, contact_tol: float) -> float:
    """run.py:454-470"""
    if contact_tol <= 0:
        return 1.0
    raw = (contact_tol - o_max) / contact_tol
    return max(0.25, min(1.0, raw))


def nudge(rad, rad_target, lmd, o_max, p: OracleParams):
    lib().orc_nudge(_ptr(rad), _ptr(rad_target), _ptr(lmd), p.n,
                    _f32(alpha_for_frames(p.adjust_frames)), _f32(p.max_step), _f32(p.r_min),
                    _f32(p.r_max), _f32(backpressure_from_overlap(o_max, p.contact_tol)),
                    p.bp_mode, _f32(p.contact_tol))


def set_threads(t: int):
    lib().orc_set_threads(int(t))


def num_threads() -> int:
    return int(lib().orc_num_threads())


# --------------------------------------------------------------- dirty tiles
def dirty_mark(pos, rad, pos_prev, rad_prev, dirty, p: OracleParams, pos_frac=0.5,
               rad_frac=0.25, halo=1):
    vs = p.L / p.R
    lib().orc_dirty_mark(_ptr(pos), _ptr(rad), _ptr(pos_prev), _ptr(rad_prev), p.n, p.R,
                         p.halfL, _f32(p.L), _f32(pos_frac * vs), _f32(rad_frac * vs), int(halo),
                         _ptr(dirty))


def dirty_count(dirty, R: int) -> int:
    return int(lib().orc_dirty_count(_ptr(dirty), int(R)))


# ------------------------------------------------------------------ topology
@dataclass
class TopoParams:
    """config.py:453-487 (topology constants)."""
    mult: float = 2.2                 # TOPO_MAX_RADIUS_MULTIPLE
    cap: int = 28                     # MAX_TOPO_NEIGHBORS
    stride: int = 3                   # TOPO_PAIR_SUBSAMPLING_STRIDE
    early_exit: bool = True           # TOPO_EARLY_EXIT_HIGH_DEGREE
    deg_high: float = 18.0            # TOPO_DEG_HIGH
    cell_size: float = 0.06           # CELL_SIZE


def topo_candidates(pos, rad, grid, p: OracleParams, tp: TopoParams):
    cc, cs, ci = grid
    pairs = np.zeros((p.n, tp.cap), np.int32)
    pc = np.zeros(p.n, np.int32)
    tr = np.zeros(p.n, np.int32)
    lib().orc_topo_candidates(_ptr(pos), _ptr(rad), _ptr(cs), _ptr(cc), _ptr(ci), p.n, p.G,
                              _f32(p.L), p.invL, p.halfL, _f32(tp.mult), tp.cap, _ptr(pairs),
                              _ptr(pc), _ptr(tr))
    return pairs, pc, tr


def topo_gabriel(pos, grid, pairs, pc, deg_ema, frame: int, p: OracleParams, tp: TopoParams):
    cc, cs, ci = grid
    deg = np.zeros(p.n, np.int32)
    lib().orc_topo_gabriel(_ptr(pos), _ptr(cs), _ptr(cc), _ptr(ci), p.n, p.G, _f32(p.L), p.invL,
                           p.halfL, _f32(tp.cell_size), int(frame), tp.stride,
                           int(tp.early_exit), _f32(tp.deg_high), tp.cap, _ptr(pairs), _ptr(pc),
                           _ptr(deg_ema), _ptr(deg))
    return deg


def topo_batched(pos, rad, grid, batch, num_batches, q, frame, pairs, pc, tr, deg,
                 p: OracleParams, tp: TopoParams):
    cc, cs, ci = grid
    lib().orc_topo_batched(_ptr(pos), _ptr(rad), _ptr(cs), _ptr(cc), _ptr(ci), p.n, p.G,
                           _f32(p.L), p.invL, p.halfL, _f32(tp.mult), _f32(tp.cell_size),
                           int(batch), int(num_batches), int(q), int(frame), tp.cap, _ptr(pairs),
                           _ptr(pc), _ptr(tr), _ptr(deg))


def topo_knn(pos, rad, grid, k: int, p: OracleParams, tp: TopoParams):
    cc, cs, ci = grid
    deg = np.zeros(p.n, np.int32)
    lib().orc_topo_knn(_ptr(pos), _ptr(rad), _ptr(cs), _ptr(cc), _ptr(ci), p.n, p.G, _f32(p.L),
                       p.invL, p.halfL, _f32(tp.mult), int(k), _ptr(deg))
    return deg


def topo_ema(deg, ema, alpha: float):
    lib().orc_topo_ema(_ptr(deg), _ptr(ema), _f32(alpha), len(deg))


def topo_radii(rad, deg_eff, lo, hi, grow, shrink, rmin, rmax):
    lib().orc_topo_radii(_ptr(rad), _ptr(deg_eff), _f32(lo), _f32(hi), _f32(grow), _f32(shrink),
                         _f32(rmin), _f32(rmax), len(rad))


# ------------------------------------------------------- run.py's JFA schedule
def skip_signals(pos_curr, pos_prev, rad_curr, rad_prev, fsc, L: float, f_low: int, f_high: int):
    """The temporal-skip signals as run.py:913-976 computes them with numpy
    (float32 arrays; pos_prev / rad_prev None on the first frame)."""
    n = len(rad_curr)
    out = {"n": n, "r_mean": float(rad_curr.mean()) if n > 0 else 0.0001}
    if pos_prev is not None and rad_prev is not None:
        dr_abs = np.abs(rad_curr - rad_prev)
        out["sigma_dr"] = float(dr_abs.std())
        d = pos_curr - pos_prev
        d = np.where(np.abs(d) > L * 0.5, d - np.sign(d) * L, d)
        out["vmax_dt"] = float(np.max(np.linalg.norm(d, axis=1)))
    else:
        out["sigma_dr"] = -1.0
        out["vmax_dt"] = -1.0
    out["fsc_mean"] = float(fsc.mean())
    out["out_of_band"] = int(np.sum((fsc < f_low) | (fsc > f_high)))
    out["zero_fsc"] = int(np.sum(fsc == 0))
    return out


@dataclass
class SkipParams:
    """config.py:158-204"""
    enabled: bool = True              # JFA_TEMPORAL_SKIP_ENABLED
    th_rsigma: float = 0.004          # TH_RSIGMA
    th_margin: float = 0.4            # TH_MARGIN_SAFE
    th_fsc_drift: float = 0.05        # TH_FSC_DRIFT
    max_skip: int = 15                # MAX_SKIP_FRAMES
    warm: int = 30                    # JFA_WARMSTART_FRAMES
    adaptive: bool = True             # JFA_ADAPTIVE_ENABLED
    vpd: float = 12.0                 # JFA_VOXELS_PER_DIAMETER
    voxel_scale: float = 2.8          # JFA_VOXEL_SCALE
    res_min: int = 192                # JFA_RES_MIN
    res_max: int = 320                # JFA_RES_MAX


class RunPySchedule:
    """run.py:898-1018 restated: the per-frame JFA decision and its state."""

    def __init__(self, sp: SkipParams):
        self.sp = sp
        self.jfa_frame_counter = 0
        self.frames_since_jfa = 0
        self.band_change_lockout = 0
        self.last_fsc_mu = None
        self.have_prev = False

    def decide(self, sig) -> tuple[bool, str]:
        sp = self.sp
        self.jfa_frame_counter += 1
        current_frame = self.jfa_frame_counter
        self.frames_since_jfa += 1
        r_mean = sig["r_mean"]
        if self.have_prev:
            sigma_dr_over_r = sig["sigma_dr"] / max(r_mean, 1e-9)
            vmax_dt = sig["vmax_dt"]
        else:
            sigma_dr_over_r = 999.0
            vmax_dt = 999.0
        delta_fsc_mu = (abs(sig["fsc_mean"] - self.last_fsc_mu)
                        if self.last_fsc_mu is not None else 999.0)
        th_margin = sp.th_margin * r_mean
        if self.band_change_lockout > 0:
            self.band_change_lockout -= 1
        t_warm = current_frame <= sp.warm
        t_watch = self.frames_since_jfa >= sp.max_skip
        t_band = self.band_change_lockout > 0
        t_act = (sigma_dr_over_r > sp.th_rsigma or vmax_dt > th_margin
                 or delta_fsc_mu > sp.th_fsc_drift)
        t_oob = False
        pct = 0.0
        if self.frames_since_jfa > 1:
            pct = float(sig["out_of_band"]) / float(max(1, sig["n"]))
            t_oob = pct > 0.10
        run = t_warm or t_watch or t_band or t_act or t_oob or not sp.enabled
        reason = ""
        if run:
            if t_warm:
                reason = "warm-start"
            elif t_band:
                reason = "band-change"
            elif t_watch:
                reason = "watchdog"
            elif t_oob:
                reason = f"out-of-band-guard ({pct * 100:.1f}%)"
            elif t_act:
                reason = "activity"
            else:
                reason = "fallback"
            self.frames_since_jfa = 0
        self.have_prev = True
        return run, reason

    def resolution(self, r_mean: float, L: float) -> int:
        """run.py:1049-1068"""
        sp = self.sp
        if sp.adaptive:
            res = int(round(L * sp.vpd / (2.0 * r_mean)))
        else:
            res = int(round(L / (sp.voxel_scale * r_mean)))
        return max(sp.res_min, min(res, sp.res_max))


# --------------------------------------------------------------- frame driver
@dataclass
class OracleSim:
    """Headless frame driver in run.py's order (run.py:699-1261), restated.

    Frame: (1) grid build; (2) max overlap; (3) settle nudge while settle > 0;
    (4) M pressure sweeps on the last JFA's face_ids/fsc; (5) Brownian jitter;
    (6) K x {grid build; PBD}; (6B) OU jitter when p.ou; (7) grid build; (8) on JFA frames: JFA, majority
    filter, faces, finalize, EMA, then the warm-start gate and set_fsc_targets.
    """
    p: OracleParams
    pos: np.ndarray
    rad: np.ndarray
    frame: int = 0
    settle: int = 0
    rad_target: np.ndarray = None
    fsc: np.ndarray = None
    ema: np.ndarray = None
    prev: np.ndarray = None
    face_ids: np.ndarray = None
    face_counts: np.ndarray = None
    nl: np.ndarray = None
    used: np.ndarray = None
    lmd: np.ndarray = None
    v_jit: np.ndarray = None
    labels: np.ndarray = None
    grid: tuple = None
    last: dict = field(default_factory=dict)

    def __post_init__(self):
        n = self.p.n
        self.pos = np.ascontiguousarray(self.pos, np.float32).reshape(n, 3).copy()
        self.rad = np.ascontiguousarray(self.rad, np.float32).copy()
        self.rad_target = self.rad.copy()
        self.fsc = np.zeros(n, np.int32)
        self.ema = np.zeros(n, np.float32)
        self.prev = np.zeros((n, S), np.float32)
        self.face_ids = np.zeros((n, S), np.int32)  # Taichi fields start zeroed
        self.face_counts = np.zeros((n, S), np.int32)
        self.nl = np.full((n, S), -1, np.int32)
        self.used = np.zeros(n, np.int32)
        self.lmd = np.zeros(n, np.float32)
        self.v_jit = np.zeros((n, 3), np.float32)  # init_jitter_velocities (run.py:346)

    def initialize(self):
        """wrap_seeded_positions + warmup_pbd (run.py:233-318)."""
        p = self.p
        w = self.pos
        w[:] = w - np.float32(p.L) * np.floor(w * np.float32(p.invL) + np.float32(0.5))
        for _ in range(p.warmup_pbd):
            self.grid = grid_build(self.pos, p)
            self.pos = pbd(self.pos, self.rad, self.grid, p)

    def run_jfa(self):
        p = self.p
        lab, ch, done = jfa_labels(self.pos, self.rad, p)
        filt = majority_filter(lab, p.R)
        self.face_ids, self.face_counts = accumulate_faces(filt, p.R, p.n)
        self.nl, self.used, self.fsc = finalize(self.rad, self.face_ids, self.face_counts,
                                                self.prev, p)
        fsc_ema(self.fsc, self.ema, p.ema_alpha)
        self.labels = lab
        self.last["changes"] = ch
        self.last["passes"] = done

    def dynamics(self):
        """Steps (1)-(7) of a frame."""
        p, f = self.p, self.frame
        self.grid = grid_build(self.pos, p)
        o_max, self.lmd = max_overlap(self.pos, self.rad, self.grid, p)
        if self.settle > 0:
            nudge(self.rad, self.rad_target, self.lmd, o_max, p)
            self.settle -= 1
        for _ in range(p.pressure_iters):
            pressure(self.rad, self.face_ids, self.fsc, f, p)
        brownian(self.pos, p, f)
        for _ in range(p.pbd_iters):
            self.grid = grid_build(self.pos, p)
            self.pos = pbd(self.pos, self.rad, self.grid, p)
        if p.ou:
            ou_jitter(self.pos, self.v_jit, self.rad, p, f)
        self.grid = grid_build(self.pos, p)
        self.last["o_max"] = o_max

    def measure(self, jfa_frame: bool):
        """Step (8) of a frame and its end."""
        p, f = self.p, self.frame
        if jfa_frame:
            self.run_jfa()
            f0 = float(np.sum(self.fsc == 0)) / float(max(1, p.n))
            warm = (f < p.warm_frames) or (f0 > p.zero_thresh)
            if not warm:
                set_targets(self.rad, self.rad_target, self.fsc, self.ema, p)
                self.settle = p.adjust_frames
        self.last["jfa"] = jfa_frame
        self.frame += 1

    def step_run_py(self, sched: RunPySchedule, state: dict) -> tuple[bool, str, int]:
        """A frame with run.py's own JFA schedule: dynamics, signals against
        the previous frame, decision, adaptive resolution, measurement.
        ``state`` carries pos_prev / rad_prev between frames."""
        p = self.p
        self.dynamics()
        sig = skip_signals(self.pos, state.get("pos_prev"), self.rad, state.get("rad_prev"),
                           self.fsc, p.L, p.f_low, p.f_high)
        run, reason = sched.decide(sig)
        state["pos_prev"] = self.pos.copy()
        state["rad_prev"] = self.rad.copy()
        if run:
            p.R = sched.resolution(sig["r_mean"], p.L)
        self.measure(run)
        if run and sched.sp.enabled:
            sched.last_fsc_mu = float(self.fsc.mean())   # run.py:1083-1085
        return run, reason, p.R

    def step(self):
        self.dynamics()
        self.measure(self.p.is_jfa_frame(self.frame))
