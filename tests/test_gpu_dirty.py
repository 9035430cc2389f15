"""Dirty tiles on the GPU (fos.jfa mark/count over fos_dirty_*) against the
oracle, bit-exact, on a foam before and after a few frames of dynamics."""
import numpy as np
import pytest
import torch

from fos import inputs, jfa, runtime
from fos.config import FosConfig
from fos.driver import FoamSim
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("frames,res", [(1, 128), (5, 96)])
def test_dirty_tiles_match_oracle(frames, res):
    foam = inputs.headline()
    sim = FoamSim.from_foam(foam)
    sim.initialize()
    sim.run(3)
    torch.cuda.synchronize()
    pp, rp = sim.pos.clone(), sim.rad.clone()
    sim.run(frames)
    torch.cuda.synchronize()
    cfg = FosConfig.for_foam(foam, JFA_RES_MIN=32, JFA_RES_MAX=128)
    runtime.configure(cfg)
    jfa.init_jfa(max_particles=foam.n, max_res=128)
    jfa.set_resolution(res)
    jfa.update_tile_cache(pp, rp, foam.n)
    jfa.clear_dirty_tiles()
    jfa.mark_dirty_tiles(sim.pos, sim.rad, foam.n)
    got = jfa.tile_dirty.to_numpy()
    cnt = jfa.count_dirty_tiles()
    p = O.OracleParams(n=foam.n, R=res)
    t = (res + 15) // 16
    want = np.zeros(t ** 3, np.uint8)
    O.dirty_mark(sim.pos.cpu().numpy(), sim.rad.cpu().numpy(), pp.cpu().numpy(), rp.cpu().numpy(),
                 want, p)
    assert got.shape == (t, t, t)
    assert np.array_equal(got.reshape(-1), want)
    assert cnt == O.dirty_count(want, res)
    jfa.clear_dirty_tiles()
    assert jfa.count_dirty_tiles() == 0
