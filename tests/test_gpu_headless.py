"""run.py's own frame flow on the GPU (fos.headless): the split frame, the
temporal-skip signals and the per-frame decisions against the oracle.

Bars:
- fos_frame_dynamics + fos_frame_measure equal fos_frame bit for bit;
- signals against numpy on the same device state (run.py:913-976): the
  largest displacement, FSC mean and band counts exact; the mean radius
  within one float32 ulp (numpy sums float32 pairwise, the library exactly);
  σ(|Δr|) within 1e-5 relative (numpy float32, the library double);
- on every frame the decision, its reason and the adaptive resolution equal
  the oracle's schedule fed those numpy signals.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from fos import inputs
from fos._lib import call
from fos.context import stream
from fos.driver import FoamSim
from fos.headless import HeadlessRun
from oracle import oracle as O

from helpers import oracle_params

pytestmark = pytest.mark.gpu
OVER = dict(JFA_RES_MIN=32, JFA_RES_MAX=96, JFA_VOXELS_PER_DIAMETER=4.0,
            JFA_WARMSTART_FRAMES=6, MAX_SKIP_FRAMES=5)


def test_split_frame_equals_frame():
    foam = inputs.small()
    a = FoamSim.from_foam(foam, use_graph=False, JFA_WARM_FRAMES=3, JFA_CADENCE=2)
    b = FoamSim.from_foam(foam, use_graph=False, JFA_WARM_FRAMES=3, JFA_CADENCE=2)
    a.initialize()
    b.initialize()
    for f in range(8):
        a.step()
        jfa = 1 if b.cfg.is_jfa_frame(f) else 0
        call("fos_frame_dynamics", b.ctx.h, C.byref(b.state), C.byref(b.fp), stream())
        call("fos_frame_measure", b.ctx.h, C.byref(b.state), C.byref(b.fp), jfa, stream())
    torch.cuda.synchronize()
    for key in ("pos", "rad", "rad_target", "fsc", "fsc_ema", "neighbor_list", "cell_indices"):
        assert torch.equal(getattr(a, key), getattr(b, key)), key
    assert a.counters() == b.counters()


def _sched(cfg):
    return O.RunPySchedule(O.SkipParams(
        enabled=cfg.JFA_TEMPORAL_SKIP_ENABLED, th_rsigma=cfg.TH_RSIGMA,
        th_margin=cfg.TH_MARGIN_SAFE, th_fsc_drift=cfg.TH_FSC_DRIFT,
        max_skip=cfg.MAX_SKIP_FRAMES, warm=cfg.JFA_WARMSTART_FRAMES,
        adaptive=cfg.JFA_ADAPTIVE_ENABLED, vpd=cfg.JFA_VOXELS_PER_DIAMETER,
        voxel_scale=cfg.JFA_VOXEL_SCALE, res_min=cfg.JFA_RES_MIN, res_max=cfg.JFA_RES_MAX))


CALM = dict(TH_RSIGMA=0.5, TH_MARGIN_SAFE=1.0, TH_FSC_DRIFT=0.5)  # lets frames skip


@pytest.mark.parametrize("over", [{}, CALM, dict(CALM, JITTER_ENABLED=True, JITTER_RMS=2.0)])
def test_signals_and_decisions_match_oracle(over):
    foam = inputs.small()
    hr = HeadlessRun.from_foam(foam, **OVER, **over)
    cfg = hr.cfg
    ref = _sched(cfg)
    hr.initialize()
    want = {}

    def check(sig):
        pos = hr.sim.pos.cpu().numpy()
        rad = hr.sim.rad.cpu().numpy()
        fsc = hr.sim.fsc.cpu().numpy()
        pp = hr.pos_prev.cpu().numpy() if hr.have_prev else None
        rp = hr.rad_prev.cpu().numpy() if hr.have_prev else None
        ns = O.skip_signals(pos, pp, rad, rp, fsc, cfg.DOMAIN_SIZE, cfg.FSC_LOW, cfg.FSC_HIGH)
        assert sig["n"] == ns["n"]
        assert sig["vmax_dt"] == ns["vmax_dt"]
        assert sig["fsc_mean"] == ns["fsc_mean"]
        assert (sig["out_of_band"], sig["zero_fsc"]) == (ns["out_of_band"], ns["zero_fsc"])
        r32 = np.float32(ns["r_mean"])
        assert abs(sig["r_mean"] - ns["r_mean"]) <= float(np.spacing(r32))
        if hr.have_prev:
            assert sig["sigma_dr"] == pytest.approx(ns["sigma_dr"], rel=1e-5, abs=1e-12)
        run, reason = ref.decide(ns)
        want["run"], want["reason"] = run, reason
        want["res"] = ref.resolution(ns["r_mean"], cfg.DOMAIN_SIZE) if run else None

    hr.on_signals = check
    runs = skips = 0
    for _ in range(40):
        rec = hr.step()
        assert (rec["jfa"], rec["reason"]) == (want["run"], want["reason"]), rec
        if rec["jfa"]:
            assert rec["res"] == want["res"] == hr.ctx.res
            ref.last_fsc_mu = float(hr.sim.fsc.cpu().numpy().mean())
            runs += 1
        else:
            skips += 1
    assert runs >= 6
    if over:
        assert skips >= 1
    assert hr.ctx.device_error() == 0


def test_first_frames_match_oracle_run():
    """Frame 0 is bit-exact end to end on both sides; with the same schedule
    and signals, the resolution and the FSC of the first run agree."""
    foam = inputs.small()
    hr = HeadlessRun.from_foam(foam, **OVER)
    hr.initialize()
    cfg = hr.cfg
    osim = O.OracleSim(oracle_params(foam), foam.pos, foam.rad)
    osim.initialize()
    sched = _sched(cfg)
    run, reason, res = osim.step_run_py(sched, {})
    rec = hr.step()
    torch.cuda.synchronize()
    assert (rec["jfa"], rec["reason"], rec["res"]) == (run, reason, res)
    assert np.array_equal(hr.sim.pos.cpu().numpy(), osim.pos)
    assert np.array_equal(hr.sim.fsc.cpu().numpy(), osim.fsc)
    assert np.array_equal(hr.sim.neighbor_list.cpu().numpy(), osim.nl)


def test_telemetry_lines():
    lines = []
    hr = HeadlessRun.from_foam(inputs.small(), log=lines.append, **OVER)
    hr.initialize()
    hr.run(14)
    text = "\n".join(lines)
    assert "[JFA Skip] Warm-start: running every frame for first 6 frames" in text
    assert "[JFA Run ] reason=warm-start | since=1" in text
    assert "[JFA Step 4] FSC μ=" in text and "res=" in text
    assert "[JFA Skip] σ(Δr)/r=" in text or "reason=activity" in text


def test_watchdog_schedule():
    hr = HeadlessRun.from_foam(inputs.small(), TH_RSIGMA=1e9, TH_MARGIN_SAFE=1e9,
                               TH_FSC_DRIFT=1e9, FSC_LOW=0, FSC_HIGH=1000, **{
                                   k: v for k, v in OVER.items() if k != "MAX_SKIP_FRAMES"},
                               MAX_SKIP_FRAMES=4)
    hr.initialize()
    hr.run(20)
    runs = [r["frame"] for r in hr.history if r["jfa"]]
    assert runs == [0, 1, 2, 3, 4, 5, 9, 13, 17]
    assert {r["reason"] for r in hr.history if r["jfa"] and r["frame"] > 5} == {"watchdog"}


def test_topology_step_runs_on_cadence():
    """run.py:1266-1280 with TOPO_ENABLED: degrees on cadence frames, EMA every frame."""
    hr = HeadlessRun.from_foam(inputs.small(), TOPO_ENABLED=True, TOPO_UPDATE_CADENCE=3, **OVER)
    hr.initialize()
    hr.run(2)
    ema1 = hr.topo["ema"].clone()
    assert torch.count_nonzero(hr.topo["deg"]).item() > 0   # frame 0 computed degrees
    hr.run(1)                                                # frame 2: EMA only
    torch.cuda.synchronize()
    deg = hr.topo["deg"].float()
    want = 0.1 * deg + (1.0 - 0.1) * ema1
    assert torch.allclose(hr.topo["ema"], want, rtol=1e-6, atol=1e-6)
