"""The reference-shaped Python surface (fos.jfa / fos.grid / fos.dynamics), driven
the way run.py drives jfa.py / grid.py / dynamics.py, against the oracle."""
import numpy as np
import pytest
import torch

from fos import inputs, runtime
from fos.config import FosConfig
from oracle import oracle as O

from helpers import oracle_params, wrapped

pytestmark = pytest.mark.gpu


def test_run_py_sequence_matches_oracle():
    foam = inputs.small()
    cfg = FosConfig.for_foam(foam, MAX_PARTICLES=2048)
    runtime.configure(cfg)
    from fos import dynamics as D
    from fos import grid as Gr
    from fos import jfa
    jfa.init_jfa(max_particles=2048, max_res=64)
    jfa.set_resolution(64)
    assert jfa.JFA_RES == 64 and jfa.JFA_NUM_PASSES == 7
    n = foam.n
    G3 = cfg.grid_res() ** 3
    pos = torch.zeros((2048, 3), dtype=torch.float32, device="cuda")
    rad = torch.zeros(2048, dtype=torch.float32, device="cuda")
    pos[:n] = torch.as_tensor(foam.pos)
    rad[:n] = torch.as_tensor(foam.rad)
    cc = torch.zeros(G3, dtype=torch.int32, device="cuda")
    cs, cw = torch.zeros_like(cc), torch.zeros_like(cc)
    ci = torch.zeros(2048, dtype=torch.int32, device="cuda")
    lmd = torch.zeros(2048, dtype=torch.float32, device="cuda")
    dr = torch.zeros(2048, dtype=torch.float32, device="cuda")
    # rebuild_grid (run.py:476-504)
    Gr.clear_grid(cc)
    Gr.count_particles_per_cell(pos, cc, n)
    Gr.prefix_sum(cc, cs)
    Gr.copy_cell_pointers(cs, cw)
    Gr.scatter_particles(pos, cw, ci, n)
    p = oracle_params(foam)
    opos = foam.pos.copy()
    grid = O.grid_build(opos, p)
    assert np.array_equal(pos[:n].cpu().numpy(), opos)
    assert np.array_equal(ci[:n].cpu().numpy(), grid[2])
    omax, olmd = O.max_overlap(opos, foam.rad, grid, p)
    assert D.compute_max_overlap(pos, rad, cs, cc, ci, lmd, n) == omax
    D.project_overlaps(pos, rad, cs, cc, ci, n)
    opos = O.pbd(opos, foam.rad, grid, p)
    assert np.array_equal(pos[:n].cpu().numpy(), opos)
    fsc_np, stats = jfa.run_jfa(pos, rad, n)
    for key in ("num_passes", "early_exit", "delta_history", "jfa_res", "voxel_size", "mean_score",
                "std_score", "valid_pairs_pct", "p_dir", "p_und_accepted", "overflow_count",
                "overflow_pct", "mean_fsc", "min_fsc", "max_fsc", "mean_fsc_ema", "fsc_ema"):
        assert key in stats
    lab, _, _ = O.jfa_labels(opos, foam.rad, p)
    ids, cnt = O.accumulate_faces(O.majority_filter(lab, p.R), p.R, n)
    prev = np.zeros((n, 32), np.float32)
    nl, used, fsc = O.finalize(foam.rad, ids, cnt, prev, p)
    assert np.array_equal(fsc_np, fsc)
    assert jfa.fsc[0] == fsc[0]
    assert np.array_equal(jfa.fsc.to_numpy()[:n], fsc)
    assert stats["p_dir"] == int(used.sum()) and stats["num_passes"] == 7
    assert abs(stats["mean_fsc"] - fsc.mean()) < 1e-5
    v = jfa.validate_jfa(n)
    assert v["passed"] and v["self_loops"] == 0
    mx, ch = D.equilibrate_pressure(n, 3, pos, rad, dr, jfa.face_ids, jfa.fsc, p.k, p.P,
                                    p.pair_cap, p.max_nei, p.r_min, p.r_max)
    orad = foam.rad.copy()
    omx, och, _ = O.pressure(orad, ids, fsc, 3, p)
    assert np.max(np.abs(rad[:n].cpu().numpy() - orad) / orad) <= 1e-5
    assert abs(ch - och) <= 2
    jfa.power_beta_current[None] = 1.0
    assert jfa.power_beta_current[None] == 1.0
    rt = torch.zeros(2048, dtype=torch.float32, device="cuda")
    D.set_fsc_targets(rad, rt, jfa.fsc, jfa.fsc_ema, n, 10, 16, 0.10, p.r_min, p.r_max)
    g, s, i, md, mxd = D.compute_controller_stats(rad, rt, jfa.fsc_ema, n, 10, 16)
    assert g + s + i == n
    jfa.mark_dirty_tiles(pos, rad, n)
    assert jfa.count_dirty_tiles() > 0
    jfa.clear_dirty_tiles()
    assert jfa.count_dirty_tiles() == 0
