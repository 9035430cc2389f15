"""run.py's JFA schedule (run.py:898-1068) as host logic: the library-side
``TemporalSkip`` / ``adaptive_resolution`` against the oracle's literal
restatement, on signal sequences that reach every trigger."""
import numpy as np
import pytest

from fos.config import FosConfig
from fos.headless import TemporalSkip, adaptive_resolution
from oracle import oracle as O


def _pair(**over):
    cfg = FosConfig(**over)
    sp = O.SkipParams(enabled=cfg.JFA_TEMPORAL_SKIP_ENABLED, th_rsigma=cfg.TH_RSIGMA,
                      th_margin=cfg.TH_MARGIN_SAFE, th_fsc_drift=cfg.TH_FSC_DRIFT,
                      max_skip=cfg.MAX_SKIP_FRAMES, warm=cfg.JFA_WARMSTART_FRAMES,
                      adaptive=cfg.JFA_ADAPTIVE_ENABLED, vpd=cfg.JFA_VOXELS_PER_DIAMETER,
                      voxel_scale=cfg.JFA_VOXEL_SCALE, res_min=cfg.JFA_RES_MIN,
                      res_max=cfg.JFA_RES_MAX)
    return cfg, TemporalSkip(cfg), O.RunPySchedule(sp)


def _drive(frames, seed, **over):
    """Both schedules on the same signals.  FSC changes only at a JFA run: the
    oracle records the new mean right after it (run.py:1083-1085), the
    library at the next frame's signals."""
    cfg, mine, ref = _pair(**over)
    rng = np.random.default_rng(seed)
    n = 1000
    fsc_now = 11.0
    out = []
    for f in range(frames):
        calm = rng.random() < 0.7
        sig = {"n": n, "r_mean": float(np.float32(rng.uniform(0.004, 0.02))),
               "sigma_dr": float(rng.uniform(0, 1e-5 if calm else 1e-3) * 0.01),
               "vmax_dt": float(rng.uniform(0, 1e-4 if calm else 1e-2)),
               "fsc_mean": fsc_now,
               "out_of_band": int(rng.integers(0, 60 if calm else 200)), "zero_fsc": 0}
        run_a, why_a, _ = mine.decide(dict(sig), f > 0)
        run_b, why_b = ref.decide(dict(sig))
        assert (run_a, why_a) == (run_b, why_b), f"frame {f}"
        if run_a:
            assert adaptive_resolution(cfg, sig["r_mean"]) == ref.resolution(sig["r_mean"],
                                                                               cfg.DOMAIN_SIZE)
            fsc_now = float(np.round(rng.uniform(9, 15), 3))
            if cfg.JFA_TEMPORAL_SKIP_ENABLED:   # run.py:1083-1085
                ref.last_fsc_mu = fsc_now
            mine.jfa_done()
        out.append((run_a, why_a))
    return out


def test_schedules_agree_and_reach_every_trigger():
    seen = set()
    for seed in range(6):
        for run, why in _drive(120, seed):
            seen.add(why.split(" ")[0] if run else "skip")
    assert {"warm-start", "activity", "out-of-band-guard", "skip"} <= seen


def test_watchdog_fires_after_max_skip_frames():
    out = _drive(60, 3, TH_RSIGMA=1e9, TH_MARGIN_SAFE=1e9, TH_FSC_DRIFT=1e9,
                 JFA_WARMSTART_FRAMES=2, MAX_SKIP_FRAMES=4)
    runs = [f for f, (r, _) in enumerate(out) if r]
    reasons = {w for r, w in out if r}
    assert runs[:2] == [0, 1]
    # out-of-band can fire too; the watchdog bounds every gap
    assert max(np.diff(runs)) <= 4
    assert "watchdog" in reasons or all(w.startswith("out-of-band") for w in reasons - {"warm-start"})


def test_skip_disabled_runs_every_frame():
    out = _drive(40, 1, JFA_TEMPORAL_SKIP_ENABLED=False)
    assert all(r for r, _ in out)


@pytest.mark.parametrize("adaptive", [True, False])
def test_adaptive_resolution_matches(adaptive):
    cfg, _, ref = _pair(JFA_ADAPTIVE_ENABLED=adaptive)
    for r in np.linspace(0.0003, 0.05, 400):
        r = float(np.float32(r))
        assert adaptive_resolution(cfg, r) == ref.resolution(r, cfg.DOMAIN_SIZE)
    # the reference configuration: L = 0.189, 12 voxels per diameter, [192, 320]
    assert adaptive_resolution(cfg, 0.006) == (192 if adaptive else 192)
    assert adaptive_resolution(cfg, 0.0035) == (320 if adaptive else 192)
