"""Checkpoint / resume and the particle CSV on the GPU.

Bar: a run saved after k frames and resumed in a fresh context continues
bit for bit like the uninterrupted run (positions, radii, targets, FSC
fields, neighbour lists, OU velocities, device counters, and for the
headless flow its JFA decisions)."""
import numpy as np
import pytest
import torch

from fos import inputs
from fos.driver import FoamSim
from fos.headless import HeadlessRun
from fos.state_io import export_frame_csv, load_checkpoint, read_csv, save_checkpoint

pytestmark = pytest.mark.gpu
KEYS = ("pos", "rad", "rad_target", "v_jit", "fsc", "fsc_ema", "face_ids", "neighbor_list",
        "cell_indices")


def _same(a, b):
    for k in KEYS:
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    assert a.counters() == b.counters()


@pytest.mark.parametrize("over", [{}, {"JITTER_ENABLED": True, "JITTER_RMS": 3.0}])
def test_foamsim_resume_is_bit_exact(tmp_path, over):
    foam = inputs.small()
    a = FoamSim.from_foam(foam, JFA_WARM_FRAMES=4, JFA_CADENCE=3, WARMSTART_FRAMES=4, **over)
    a.initialize()
    a.run(9)   # the controller has set targets and the settle counter is running
    path = save_checkpoint(str(tmp_path / "ck.npz"), a)
    b = load_checkpoint(path)
    assert b.frame == a.frame == 9
    _same(a, b)
    for _ in range(8):
        assert a.step() == b.step()
    torch.cuda.synchronize()
    _same(a, b)


def test_headless_resume_is_bit_exact(tmp_path):
    over = dict(JFA_RES_MIN=32, JFA_RES_MAX=96, JFA_VOXELS_PER_DIAMETER=4.0,
                JFA_WARMSTART_FRAMES=4, MAX_SKIP_FRAMES=5, TH_RSIGMA=0.5, TH_MARGIN_SAFE=1.0,
                TH_FSC_DRIFT=0.5)
    a = HeadlessRun.from_foam(inputs.small(), **over)
    a.initialize()
    a.run(7)
    path = save_checkpoint(str(tmp_path / "hk.npz"), a)
    b = load_checkpoint(path)
    for _ in range(10):
        ra, rb = a.step(), b.step()
        assert (ra["jfa"], ra["reason"], ra["res"]) == (rb["jfa"], rb["reason"], rb["res"])
    torch.cuda.synchronize()
    _same(a.sim, b.sim)


def test_frame_csv_matches_device_state(tmp_path):
    sim = FoamSim.from_foam(inputs.small())
    sim.initialize()
    sim.run(3)
    path = export_frame_csv(sim, str(tmp_path))
    assert path.endswith("particle_data_frame_3.csv")
    back = read_csv(path)
    assert np.array_equal(back["pos"], sim.pos.cpu().numpy())
    assert np.array_equal(back["rad"], sim.rad.cpu().numpy())
    assert np.array_equal(back["fsc"], sim.fsc.cpu().numpy())
