"""Simulation constants, named as in the reference's config.py and jfa.py.

The reference reads these as module globals that Taichi bakes into kernels at
first compile (config.py; jfa.py:53-97).  Here they are fields of
``FosConfig``, turned into the C ABI's ``FosParams`` / ``FosFrameParams``
(include/fos.h).  Python floats stay doubles across the ABI; the library folds
them to float32 exactly as Taichi folds a Python float into a kernel literal.

``FosConfig.for_foam`` applies a workload's overrides (box L = 1, JFA
resolution, PBD / pressure iteration counts, FSC band, cadence, jitter).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace

from ._lib import FosFrameParams, FosParams


@dataclass
class FosConfig:
    DOMAIN_SIZE: float = 0.189            # config.py:21
    CELL_SIZE: float | None = None        # None -> GRID_RES given directly
    GRID_RES: int = 3                     # config.py:317
    POWER_BETA: float = 1.0               # config.py:143
    JFA_RES: int = 128                    # jfa.py:80
    JFA_RES_MIN: int = 192                # config.py:156
    JFA_RES_MAX: int = 320                # config.py:157
    JFA_EARLY_EXIT_ENABLED: bool = True   # config.py:208
    TH_PASS_DELTA: float = 0.006          # config.py:209
    MIN_JFA_PASSES: int = 3               # config.py:210
    TIE_LOWER_INDEX: bool = False         # north-star tie rule; reference = scan order
    EXPECTED_FACE_SCALE: float = 1.5      # jfa.py:58
    T_ADD: float = 0.15                   # jfa.py:63
    T_DROP: float = 0.10                  # jfa.py:64
    JFA_EMA_ALPHA: float = 0.33           # config.py:81
    MAX_PARTICLES: int = 50000            # jfa.py:67
    GAP_FRACTION: float = 0.015           # config.py:353
    MAX_DISPLACEMENT_FRAC: float = 0.2    # config.py:349
    DISPLACEMENT_MULTIPLIER: float = 2.0  # config.py:350
    EPS: float = 1e-8                     # config.py:324
    CONTACT_TOL: float = 0.035            # config.py:254
    FSC_DEADBAND: float = 1.0             # config.py:100
    FSC_LOW: int = 8                      # config.py:90
    FSC_HIGH: int = 20                    # config.py:91
    GROWTH_PCT: float = 0.10              # config.py:92
    ADJUSTMENT_FRAMES: int = 15           # config.py:93
    MAX_STEP_PCT: float = 0.12            # config.py:96
    BACKPRESSURE_MODE: str = "local"      # config.py:101
    WARMSTART_FRAMES: int = 30            # config.py:129
    FSC_ZERO_RATE_THRESH: float = 0.10    # config.py:130
    PRESSURE_K: float = 0.10              # config.py:112
    PRESSURE_EXP: float = 3.0             # config.py:113
    PRESSURE_PAIR_CAP: float = 0.02       # config.py:114
    MAX_EQ_NEI: int = 10                  # config.py:115
    BROWNIAN_STRENGTH: float = 0.0002     # config.py:123
    R_MIN: float = 0.002                  # config.py:49
    R_MAX: float = 0.010                  # config.py:50
    PBD_BASE_PASSES: int = 4              # config.py:342
    # OU velocity jitter after the PBD sweeps (run.py:855-867).  config.py:493
    # has it on; the headless workloads run with the Brownian channel only.
    JITTER_ENABLED: bool = False
    JITTER_RMS: float = 0.10              # config.py:494
    JITTER_TAU: float = 1.0               # config.py:496
    DT: float = 0.016                     # config.py:400
    MAX_DRIFT_FRACTION: float = 0.20      # config.py:498
    # run.py's own JFA schedule (fos.headless): temporal skip and adaptive
    # resolution (run.py:898-1068)
    JFA_TEMPORAL_SKIP_ENABLED: bool = True  # config.py:200
    TH_RSIGMA: float = 0.004              # config.py:201
    TH_MARGIN_SAFE: float = 0.4           # config.py:202
    TH_FSC_DRIFT: float = 0.05            # config.py:203
    MAX_SKIP_FRAMES: int = 15             # config.py:204
    JFA_WARMSTART_FRAMES: int = 30        # config.py:173
    JFA_ADAPTIVE_ENABLED: bool = True     # config.py:163
    JFA_VOXELS_PER_DIAMETER: float = 12.0  # config.py:164
    JFA_VOXEL_SCALE: float = 2.8          # config.py:158
    # warm-started JFA (no reference counterpart): first step of its pass
    # schedule; FoamSim uses it on JFA frames when jfa_warm is set
    JFA_WARM_STEP: int = 4
    # dirty-tile bookkeeping of the JFA grid (config.py:181-191)
    JFA_DIRTY_TILES_ENABLED: bool = True
    JFA_TILE_SIZE: int = 16
    JFA_DIRTY_HALO: int = 1
    JFA_DIRTY_WARMSTART: bool = True
    JFA_DIRTY_POS_THRESHOLD: float = 0.5
    JFA_DIRTY_RAD_THRESHOLD: float = 0.25
    # topological degree (topology.py), off in the reference (config.py:453-487)
    TOPO_ENABLED: bool = False
    TOPO_UPDATE_CADENCE: int = 60
    TOPO_EMA_ALPHA: float = 0.1
    TOPO_BATCHES: int = 12
    TOPO_PAIR_SUBSAMPLE_Q: int = 3
    TOPO_DEG_LOW: int = 10
    TOPO_DEG_HIGH: int = 18
    TOPO_MAX_RADIUS_MULTIPLE: float = 2.2
    MAX_TOPO_NEIGHBORS: int = 28
    TOPO_PAIR_SUBSAMPLING_STRIDE: int = 3
    TOPO_EARLY_EXIT_HIGH_DEGREE: bool = True
    USE_KNN_TOPO: bool = False
    KNN_TOPO_K: int = 14
    # per-frame schedule of the headless driver
    PBD_ITERS: int = 4
    PRESSURE_ITERS: int = 1
    JFA_WARM_FRAMES: int = 20             # JFA every frame for the first frames
    JFA_CADENCE: int = 5                  # config.py:172, then every k-th frame
    SEED: int = 0

    def grid_res(self) -> int:
        if self.CELL_SIZE is None:
            return int(self.GRID_RES)
        return max(3, int(math.ceil(self.DOMAIN_SIZE / self.CELL_SIZE)))  # config.py:317

    def jfa_num_passes(self, res: int | None = None) -> int:
        import numpy as np
        r = self.JFA_RES if res is None else res
        return int(np.ceil(np.log2(r))) + 1  # jfa.py:223

    def cell_size(self) -> float:
        """CELL_SIZE as the topology stencil uses it (config.py:317); with
        GRID_RES given directly, the grid's own cell L / GRID_RES."""
        return float(self.CELL_SIZE) if self.CELL_SIZE is not None else \
            float(self.DOMAIN_SIZE) / float(self.GRID_RES)

    def bp_mode(self) -> int:
        return {"local": 2, "global": 1}.get(self.BACKPRESSURE_MODE, 0)

    def is_jfa_frame(self, frame: int) -> bool:
        return frame < self.JFA_WARM_FRAMES or frame % self.JFA_CADENCE == 0

    def params(self) -> FosParams:
        return FosParams(
            domain_size=float(self.DOMAIN_SIZE), grid_res=self.grid_res(),
            power_beta=float(self.POWER_BETA), early_exit=int(bool(self.JFA_EARLY_EXIT_ENABLED)),
            min_jfa_passes=int(self.MIN_JFA_PASSES), th_pass_delta=float(self.TH_PASS_DELTA),
            tie_lower_index=int(bool(self.TIE_LOWER_INDEX)),
            expected_face_scale=float(self.EXPECTED_FACE_SCALE), t_add=float(self.T_ADD),
            t_drop=float(self.T_DROP), ema_alpha=float(self.JFA_EMA_ALPHA),
            gap_fraction=float(self.GAP_FRACTION),
            max_displacement_frac=float(self.MAX_DISPLACEMENT_FRAC),
            displacement_multiplier=float(self.DISPLACEMENT_MULTIPLIER), eps=float(self.EPS),
            contact_tol=float(self.CONTACT_TOL), fsc_deadband=float(self.FSC_DEADBAND))

    def frame_params(self) -> FosFrameParams:
        return FosFrameParams(
            pbd_iters=int(self.PBD_ITERS), pressure_iters=int(self.PRESSURE_ITERS),
            f_low=int(self.FSC_LOW), f_high=int(self.FSC_HIGH),
            growth_pct=float(self.GROWTH_PCT), max_step_pct=float(self.MAX_STEP_PCT),
            adjustment_frames=int(self.ADJUSTMENT_FRAMES), bp_mode=self.bp_mode(),
            warmstart_frames=int(self.WARMSTART_FRAMES),
            zero_rate_thresh=float(self.FSC_ZERO_RATE_THRESH), r_min=float(self.R_MIN),
            r_max=float(self.R_MAX), pressure_k=float(self.PRESSURE_K),
            pressure_exp=float(self.PRESSURE_EXP), pressure_pair_cap=float(self.PRESSURE_PAIR_CAP),
            max_eq_nei=int(self.MAX_EQ_NEI), brownian_strength=float(self.BROWNIAN_STRENGTH),
            seed=int(self.SEED) & 0xFFFFFFFFFFFFFFFF, warmup_pbd=int(self.PBD_BASE_PASSES),
            ou_jitter=int(bool(self.JITTER_ENABLED)), jitter_rms=float(self.JITTER_RMS),
            jitter_tau=float(self.JITTER_TAU), dt=float(self.DT),
            max_drift_fraction=float(self.MAX_DRIFT_FRACTION),
            jfa_warm_step=int(self.JFA_WARM_STEP))

    @classmethod
    def for_foam(cls, foam, **over) -> "FosConfig":
        """Workload overrides: L = 1, JFA res as given (no [192, 320] clamp),
        hash cell 2*r_max, full JFA pass schedule (early exit off), Brownian
        strength 1e-4, the foam's band, iteration counts and cadence."""
        cfg = cls(
            DOMAIN_SIZE=1.0, CELL_SIZE=2.0 * foam.r_max, JFA_RES=foam.res,
            JFA_RES_MIN=2, JFA_RES_MAX=max(foam.res, 2), JFA_EARLY_EXIT_ENABLED=False,
            FSC_LOW=foam.f_low, FSC_HIGH=foam.f_high, R_MIN=foam.r_min, R_MAX=foam.r_max,
            PBD_ITERS=foam.pbd_iters, PRESSURE_ITERS=foam.pressure_iters,
            JFA_WARM_FRAMES=foam.jfa_warm, JFA_CADENCE=foam.jfa_cadence,
            BROWNIAN_STRENGTH=1e-4, SEED=foam.seed, MAX_PARTICLES=foam.n)
        return replace(cfg, **over)
