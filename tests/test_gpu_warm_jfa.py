"""Warm-started JFA (fos_jfa_warm; no reference counterpart): measured
agreement with the exact JFA on the same positions, and a run with it.

Bars (measured on the headline foam, stated here):
- from the same relaxed state, the warm start (previous owner grid, seeds
  re-planted, steps 4, 2, 1, 1) gives the exact run's owner label on
  >= 99.5% of voxels and the same FSC on >= 99% of particles;
- a 60-frame run with warm starts keeps the FSC histogram within 0.05 total
  variation of the exact run's and the mean FSC within 0.3.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from fos import inputs
from fos._lib import call
from fos.context import stream
from fos.driver import FoamSim

pytestmark = pytest.mark.gpu
FIELDS = ("fsc", "fsc_ema", "face_ids", "face_counts", "neighbor_list", "neighbor_used_count",
          "neighbor_prev_scores")


def _snapshot(ctx):
    return {k: getattr(ctx, k).clone() for k in FIELDS}


def _restore(ctx, snap):
    for k, v in snap.items():
        getattr(ctx, k).copy_(v)


def _jfa(sim, warm_step):
    ctx, n = sim.ctx, sim.n
    if warm_step:
        call("fos_jfa_warm", ctx.h, C.c_void_p(sim.pos.data_ptr()), C.c_void_p(sim.rad.data_ptr()),
             n, warm_step, stream())
    else:
        ctx.jfa_init(sim.pos, sim.rad, n)
        ctx.jfa_passes(n)
    lab = ctx.labels().clone()
    ctx.majority_filter()
    ctx.accumulate_faces(n)
    ctx.finalize(sim.rad, n)
    torch.cuda.synchronize()
    return lab, sim.fsc.clone()


@pytest.mark.parametrize("step", [4, 8])
def test_warm_start_agrees_with_exact(step):
    sim = FoamSim.from_foam(inputs.headline())
    sim.initialize()
    sim.run(35)            # frames 0..34: the last JFA ran on frame 30, four frames back
    torch.cuda.synchronize()
    snap = _snapshot(sim.ctx)
    lab_w, fsc_w = _jfa(sim, step)   # starts from frame 30's owner grid
    _restore(sim.ctx, snap)
    lab_x, fsc_x = _jfa(sim, 0)      # the exact JFA of the same positions
    vox = (lab_w == lab_x).float().mean().item()
    agree = (fsc_w == fsc_x).float().mean().item()
    assert vox >= 0.995, vox
    assert agree >= 0.99, agree


def test_warm_run_tracks_exact_run():
    foam = inputs.headline()
    a = FoamSim.from_foam(foam)
    b = FoamSim.from_foam(foam, jfa_warm=True)
    for s in (a, b):
        s.initialize()
        s.run(60)
    torch.cuda.synchronize()
    fa, fb = a.fsc.cpu().numpy(), b.fsc.cpu().numpy()
    ha = np.bincount(fa, minlength=40)[:40] / len(fa)
    hb = np.bincount(fb, minlength=40)[:40] / len(fb)
    assert 0.5 * np.abs(ha - hb).sum() <= 0.05
    assert abs(fa.mean() - fb.mean()) <= 0.3
    assert b.ctx.device_error() == 0


def test_warm_start_agreement_over_a_run():
    """On every JFA frame of a 100-frame exact run, the warm start from the
    previous JFA frame's owner grid is compared with the exact JFA of the same
    positions (split frame: dynamics, then both JFAs from the same fields).
    Measured on the headline foam: identical on >= 99.9% of voxels and >= 99.5%
    of particles' FSC on every JFA frame."""
    sim = FoamSim.from_foam(inputs.headline())
    sim.initialize()
    st, fp = C.byref(sim.state), C.byref(sim.fp)
    worst_vox, worst_fsc, compared = 1.0, 1.0, 0
    for f in range(100):
        jfa = sim.cfg.is_jfa_frame(f)
        call("fos_frame_dynamics", sim.ctx.h, st, fp, stream())
        if jfa and f > 0:
            snap = _snapshot(sim.ctx)
            lab_w, fsc_w = _jfa(sim, sim.cfg.JFA_WARM_STEP)
            _restore(sim.ctx, snap)
            call("fos_frame_measure", sim.ctx.h, st, fp, 1, stream())
            torch.cuda.synchronize()
            lab_x, fsc_x = sim.ctx.labels(), sim.fsc
            worst_vox = min(worst_vox, (lab_w == lab_x).float().mean().item())
            worst_fsc = min(worst_fsc, (fsc_w == fsc_x).float().mean().item())
            compared += 1
        else:
            call("fos_frame_measure", sim.ctx.h, st, fp, 1 if jfa else 0, stream())
    assert compared >= 30
    assert worst_vox >= 0.999, worst_vox
    assert worst_fsc >= 0.995, worst_fsc
