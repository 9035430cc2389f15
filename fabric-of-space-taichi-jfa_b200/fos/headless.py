"""run.py's own headless frame flow on libfos: temporal skip, adaptive JFA
resolution, OU jitter, the optional topological degree and the telemetry
lines.

``FoamSim`` runs the workloads' fixed schedule (JFA on warm-start frames, then
every k-th frame).  The reference's ``run.py`` decides instead, frame by
frame, after the dynamics (run.py:898-1018):

- activity signals against the previous frame: σ(|Δr|)/r_mean, the largest
  periodic displacement, and the drift of mean FSC since the last JFA;
- triggers: warm start (first JFA_WARMSTART_FRAMES frames), watchdog
  (MAX_SKIP_FRAMES frames since the last JFA), band-change lockout, activity
  above TH_RSIGMA / TH_MARGIN_SAFE·r_mean / TH_FSC_DRIFT, and more than 10% of
  particles out of the FSC band after a skipped frame;
- on a JFA frame the resolution follows the mean radius (run.py:1049-1068):
  JFA_VOXELS_PER_DIAMETER voxels across a mean diameter, clamped to
  [JFA_RES_MIN, JFA_RES_MAX].

``HeadlessRun`` does that with the frame split in two library calls
(``fos_frame_dynamics`` / ``fos_frame_measure``).  Between them one small
reduction (``fos_skip_signals``) computes the signals on the device, and one
64-byte read brings them to the host, where the decision is made.  The
reference instead copies positions, radii and FSC to the host every frame.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import FosSkipSignals, call
from .config import FosConfig
from .context import Context, stream
from .driver import FoamSim


class TemporalSkip:
    """The JFA decision of run.py:898-1018, with its state across frames.

    ``decide`` takes the frame's signals (FosSkipSignals fields as a dict) and
    returns (run, reason, info).  ``jfa_done`` records a JFA run, whose FSC
    mean becomes the drift baseline (run.py:1081-1085): FSC changes only in
    a JFA, so the baseline is the FSC mean the next frame's signals report."""

    def __init__(self, cfg: FosConfig):
        self.cfg = cfg
        self.counter = 0           # jfa_frame_counter
        self.since = 0             # frames_since_jfa
        self.lockout = 0           # band_change_lockout (GUI band edits only)
        self.last_fsc_mu = None
        self._baseline_pending = False

    def jfa_done(self):
        if self.cfg.JFA_TEMPORAL_SKIP_ENABLED:
            self._baseline_pending = True

    def decide(self, sig: dict, have_prev: bool) -> tuple[bool, str, dict]:
        cfg = self.cfg
        if self._baseline_pending:
            self.last_fsc_mu = sig["fsc_mean"]
            self._baseline_pending = False
        self.counter += 1
        self.since += 1
        n = sig["n"]
        r_mean = sig["r_mean"] if n > 0 else 0.0001
        if have_prev:
            sigma_dr_over_r = sig["sigma_dr"] / max(r_mean, 1e-9)
            vmax_dt = sig["vmax_dt"]
        else:
            sigma_dr_over_r = 999.0
            vmax_dt = 999.0
        if self.last_fsc_mu is not None:
            delta_fsc_mu = abs(sig["fsc_mean"] - self.last_fsc_mu)
        else:
            delta_fsc_mu = 999.0
        th_sigma = cfg.TH_RSIGMA
        th_margin = cfg.TH_MARGIN_SAFE * r_mean
        if self.lockout > 0:
            self.lockout -= 1
        warm = self.counter <= cfg.JFA_WARMSTART_FRAMES
        watchdog = self.since >= cfg.MAX_SKIP_FRAMES
        band = self.lockout > 0
        activity = (sigma_dr_over_r > th_sigma or vmax_dt > th_margin
                    or delta_fsc_mu > cfg.TH_FSC_DRIFT)
        oob_pct = 0.0
        if self.since > 1:
            oob_pct = float(sig["out_of_band"]) / float(max(1, n))
            out_of_band = oob_pct > 0.10
        else:
            out_of_band = False
        run = (warm or watchdog or band or activity or out_of_band
               or not cfg.JFA_TEMPORAL_SKIP_ENABLED)
        if not run:
            reason = ""
        elif warm:
            reason = "warm-start"
        elif band:
            reason = "band-change"
        elif watchdog:
            reason = "watchdog"
        elif out_of_band:
            reason = f"out-of-band-guard ({oob_pct * 100:.1f}%)"
        elif activity:
            reason = "activity"
        else:
            reason = "fallback"
        info = {"frame_counter": self.counter, "since": self.since,
                "sigma_dr_over_r": sigma_dr_over_r, "vmax_dt": vmax_dt,
                "delta_fsc_mu": delta_fsc_mu, "th_sigma": th_sigma, "th_margin": th_margin}
        if run:
            self.since = 0
        return run, reason, info


def adaptive_resolution(cfg: FosConfig, r_mean: float) -> int:
    """Resolution for a JFA run (run.py:1049-1068)."""
    if cfg.JFA_ADAPTIVE_ENABLED:
        res = int(round(cfg.DOMAIN_SIZE * cfg.JFA_VOXELS_PER_DIAMETER / (2.0 * r_mean)))
    else:
        res = int(round(cfg.DOMAIN_SIZE / (cfg.JFA_VOXEL_SCALE * r_mean)))
    return max(cfg.JFA_RES_MIN, min(res, cfg.JFA_RES_MAX))


class HeadlessRun:
    """run.py's frame loop without the window: FoamSim's state and frame, with
    the JFA decided per frame by ``TemporalSkip`` and the resolution by
    ``adaptive_resolution``.  ``log`` (e.g. ``print``) receives run.py's
    telemetry lines; None keeps the run silent and free of the extra syncs
    the JFA statistics need."""

    def __init__(self, cfg: FosConfig, pos, rad, device: int | None = None, log=None):
        n = int(rad.shape[0])
        max_res = max(int(cfg.JFA_RES), int(cfg.JFA_RES_MAX))
        self.cfg = cfg
        self.log = log
        self.ctx = Context(cfg, max_n=n, max_res=max_res, device=device)
        self.sim = FoamSim(cfg, pos, rad, use_graph=False, ctx=self.ctx)
        self.pos_prev = torch.empty_like(self.sim.pos)
        self.rad_prev = torch.empty_like(self.sim.rad)
        self.have_prev = False
        self.skip = TemporalSkip(cfg)
        self.frame = 0
        self.res = int(cfg.JFA_RES)
        self.history: list[dict] = []
        self.on_signals = None     # optional callback(sig) before each decision
        self.topo = None
        if cfg.TOPO_ENABLED:       # topology.allocate_fields (run.py:199)
            dev = self.sim.pos.device
            cap = int(cfg.MAX_TOPO_NEIGHBORS)
            self.topo = {"deg": torch.zeros(n, dtype=torch.int32, device=dev),
                         "ema": torch.zeros(n, dtype=torch.float32, device=dev),
                         "pairs": torch.zeros((n, cap), dtype=torch.int32, device=dev),
                         "count": torch.zeros(n, dtype=torch.int32, device=dev),
                         "trunc": torch.zeros(n, dtype=torch.int32, device=dev)}

    @classmethod
    def from_foam(cls, foam, log=None, **over) -> "HeadlessRun":
        return cls(FosConfig.for_foam(foam, **over), foam.pos, foam.rad, log=log)

    def initialize(self, frame0: int = 0):
        self.sim.initialize(frame0)
        self.frame = int(frame0)

    def signals(self, prev: bool = True) -> dict:
        sim = self.sim
        out = FosSkipSignals()
        pp = self.pos_prev.data_ptr() if prev else None
        rp = self.rad_prev.data_ptr() if prev else None
        call("fos_skip_signals", self.ctx.h, C.byref(sim.state), pp, rp, int(self.cfg.FSC_LOW),
             int(self.cfg.FSC_HIGH), C.byref(out), stream())
        return {k: getattr(out, k) for k, _ in FosSkipSignals._fields_ if k != "pad"}

    def step(self) -> dict:
        sim, cfg = self.sim, self.cfg
        call("fos_frame_dynamics", self.ctx.h, C.byref(sim.state), C.byref(sim.fp), stream())
        sig = self.signals(self.have_prev)
        if self.on_signals:
            self.on_signals(sig)
        run, reason, info = self.skip.decide(sig, self.have_prev)
        self.pos_prev.copy_(sim.pos)
        self.rad_prev.copy_(sim.rad)
        self.have_prev = True
        if self.log:
            self._log_decision(run, reason, info)
        if run:
            res = adaptive_resolution(cfg, sig["r_mean"])
            if res != self.ctx.res:
                self.ctx.set_resolution(res)
            self.res = res
        call("fos_frame_measure", self.ctx.h, C.byref(sim.state), C.byref(sim.fp), int(run),
             stream())
        if run:
            self.skip.jfa_done()
            if self.log:
                self._log_jfa()
        if self.topo is not None:
            self._topology()
        rec = {"frame": self.frame, "jfa": run, "reason": reason, "res": self.res} | info
        self.history.append(rec)
        self.frame += 1
        sim.frame = self.frame
        return rec

    def run(self, frames: int):
        for _ in range(frames):
            self.step()

    def _topology(self):
        """run.py:1266-1280: every TOPO_UPDATE_CADENCE frames the Gabriel
        degree on the frame's final grid, every frame its EMA."""
        cfg, sim, t = self.cfg, self.sim, self.topo
        g = (C.c_void_p(sim.cell_start.data_ptr()), C.c_void_p(sim.cell_count.data_ptr()),
             C.c_void_p(sim.cell_indices.data_ptr()))
        cap = int(cfg.MAX_TOPO_NEIGHBORS)
        if self.frame % cfg.TOPO_UPDATE_CADENCE == 0:
            call("fos_topo_candidates", self.ctx.h, C.c_void_p(sim.pos.data_ptr()),
                 C.c_void_p(sim.rad.data_ptr()), *g, sim.n, float(cfg.TOPO_MAX_RADIUS_MULTIPLE),
                 cap, C.c_void_p(t["pairs"].data_ptr()), C.c_void_p(t["count"].data_ptr()),
                 C.c_void_p(t["trunc"].data_ptr()), stream())
            call("fos_topo_gabriel", self.ctx.h, C.c_void_p(sim.pos.data_ptr()), *g, sim.n,
                 int(self.frame), cfg.cell_size(), int(cfg.TOPO_PAIR_SUBSAMPLING_STRIDE),
                 int(bool(cfg.TOPO_EARLY_EXIT_HIGH_DEGREE)), float(cfg.TOPO_DEG_HIGH), cap,
                 C.c_void_p(t["pairs"].data_ptr()), C.c_void_p(t["count"].data_ptr()),
                 C.c_void_p(t["ema"].data_ptr()), C.c_void_p(t["deg"].data_ptr()), stream())
        call("fos_topo_ema", self.ctx.h, C.c_void_p(t["deg"].data_ptr()),
             C.c_void_p(t["ema"].data_ptr()), float(cfg.TOPO_EMA_ALPHA), sim.n, stream())

    # ------------------------------------------------------------- telemetry
    def _log_decision(self, run, reason, info):
        cfg = self.cfg
        if run:
            if reason == "warm-start" and info["frame_counter"] == 1:
                self.log(f"[JFA Skip] Warm-start: running every frame for first "
                         f"{cfg.JFA_WARMSTART_FRAMES} frames")
            self.log(f"[JFA Run ] reason={reason} | since={info['since']}")
        else:
            self.log(f"[JFA Skip] σ(Δr)/r={info['sigma_dr_over_r']:.4f} ≤ {info['th_sigma']:.4f} | "
                     f"vmax*dt={info['vmax_dt']:.6f} ≤ {info['th_margin']:.6f} | "
                     f"ΔμFSC={info['delta_fsc_mu']:.3f} ≤ {cfg.TH_FSC_DRIFT:.3f} | "
                     f"since={info['since']}/{cfg.MAX_SKIP_FRAMES}")

    def _log_jfa(self):
        sim, n = self.sim, self.sim.n
        st = self.ctx.jfa_stats(n, sim.rad)
        val = self.ctx.validate(n)
        asym = 100.0 * val["asymmetric_pairs"] / max(1, n)
        self.log(f"[JFA Step 4] FSC μ={st['mean_fsc']:.1f} [{st['min_fsc']},{st['max_fsc']}] | "
                 f"EMA μ={st['mean_fsc_ema']:.1f}")
        self.log(f"      score: μ={st['mean_score']:.2f} σ={st['std_score']:.2f} | "
                 f"pairs: {st['p_und_accepted']} (P_dir={st['p_dir']})")
        self.log(f"      asym={asym:.1f}% overflow={st['overflow_pct']:.1f}% | "
                 f"res={self.res}³ | passes={st['num_passes']}/{self.ctx.num_passes} "
                 f"(early_exit={st['early_exit']})")
