"""The CUDA path against golden fixtures of the reference's own execution.

Each test makes, through the reference-shaped drop-in modules (fos.jfa,
fos.grid, fos.dynamics over libfos's C ABI), the same calls that
tests/golden/make_golden.py made on the unmodified reference modules, on the
same inputs, and compares the outputs:

- bit-exact: owner labels, filtered labels, face rows in slot order,
  neighbour lists, FSC, EMA and hysteresis scores over consecutive runs, the
  pass count and per-pass changes, cell lists, PBD sweeps, overlap depths,
  the controller, Brownian and OU jitter and the dirty tiles;
- within 1e-5 relative: radii after pressure sweeps (the GPU's powers for
  P = 3 against libm powf).
"""
import json
import os

import numpy as np
import pytest
import torch

from fos import runtime
from fos.config import FosConfig

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PRESSURE_RTOL = 1e-5


def load(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    return {k: z[k] for k in z.files}, json.loads(str(z["meta"]))


def setup(max_n: int, max_res: int = 32, **cfg):
    runtime.configure(FosConfig(JFA_RES=max_res, JFA_RES_MIN=8, JFA_RES_MAX=max_res,
                                MAX_PARTICLES=max_n, **cfg))
    from fos import jfa
    jfa.init_jfa(max_particles=max_n, max_res=max_res)
    return jfa


def cuda(a, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).cuda()


@pytest.mark.parametrize("case", ["jfa_r16_hysteresis", "jfa_r24_ties_early_exit",
                                  "jfa_r16_domain0189", "jfa_r24_overflow"])
def test_jfa_runs_match_reference(case):
    f, m = load(case)
    n, R = m["n"], m["R"]
    jfa = setup(n, max(32, R), DOMAIN_SIZE=m["L"], JFA_EARLY_EXIT_ENABLED=m["early_exit"],
                TH_PASS_DELTA=m.get("th_delta", 0.006), T_ADD=m.get("t_add", 0.15),
                T_DROP=m.get("t_drop", 0.10))
    jfa.set_resolution(R)
    ctx = runtime.ctx()
    for k in range(m["runs"]):
        fsc, stats = jfa.run_jfa(cuda(f[f"run{k}_pos"]), cuda(f[f"run{k}_rad"]), n)
        torch.cuda.synchronize()
        assert stats["num_passes"] == f[f"run{k}_stat_num_passes"]
        changes = np.array([round(d * R ** 3) for d in stats["delta_history"]], np.int64)
        assert np.array_equal(changes, f[f"run{k}_stat_changes"])
        assert np.array_equal(ctx.labels().cpu().numpy().reshape(-1), f[f"run{k}_labels"])
        assert np.array_equal(ctx.label_filtered().cpu().numpy().reshape(-1),
                              f[f"run{k}_filtered"])
        for name, ref in (("face_ids", "face_ids"), ("face_counts", "face_counts"),
                          ("neighbor_list", "neighbor_list"),
                          ("neighbor_used_count", "neighbor_used_count"),
                          ("fsc_ema", "fsc_ema"), ("neighbor_prev_scores", "prev_scores")):
            got = getattr(jfa, name).to_numpy()[:n]
            assert np.array_equal(got, f[f"run{k}_{ref}"]), f"run {k}: {name}"
        assert np.array_equal(fsc, f[f"run{k}_fsc"]), f"run {k}: fsc"
        assert stats["p_dir"] == f[f"run{k}_stat_p_dir"]
        assert stats["overflow_count"] == f[f"run{k}_stat_overflow_count"]
        assert stats["min_fsc"] == f[f"run{k}_stat_min_fsc"]
        assert stats["max_fsc"] == f[f"run{k}_stat_max_fsc"]
        v = jfa.validate_jfa(n)
        want = f[f"run{k}_validate"]
        assert (int(v["passed"]), v["asymmetric_pairs"], v["overflow_count"],
                v["self_loops"]) == tuple(int(x) for x in want)


@pytest.mark.parametrize("case", ["grid_g3", "grid_g5"])
def test_grid_build_matches_reference(case):
    f, m = load(case)
    n, G = m["n"], m["G"]
    setup(n, DOMAIN_SIZE=m["L"], GRID_RES=G)
    from fos import grid as Gr
    pos = cuda(f["pos"])
    cc = torch.zeros(G ** 3, dtype=torch.int32, device="cuda")
    cs, cw = torch.zeros_like(cc), torch.zeros_like(cc)
    ci = torch.zeros(n, dtype=torch.int32, device="cuda")
    Gr.clear_grid(cc)
    Gr.count_particles_per_cell(pos, cc, n)
    Gr.prefix_sum(cc, cs)
    Gr.copy_cell_pointers(cs, cw)
    Gr.scatter_particles(pos, cw, ci, n)
    assert np.array_equal(pos.cpu().numpy(), f["pos_wrapped"])
    assert np.array_equal(cc.cpu().numpy(), f["cell_count"])
    assert np.array_equal(cs.cpu().numpy(), f["cell_start"])
    assert np.array_equal(ci.cpu().numpy(), f["cell_indices"])


def test_pbd_and_max_overlap_match_reference():
    f, m = load("pbd_g4")
    n, G = m["n"], m["G"]
    setup(n, DOMAIN_SIZE=m["L"], GRID_RES=G)
    from fos import dynamics as D
    from fos import grid as Gr
    pos, rad = cuda(f["pos"]), cuda(f["rad"])
    cc = torch.zeros(G ** 3, dtype=torch.int32, device="cuda")
    cs = torch.zeros_like(cc)
    ci = torch.zeros(n, dtype=torch.int32, device="cuda")
    lmd = torch.zeros(n, dtype=torch.float32, device="cuda")
    Gr.rebuild_grid(pos, n, cc, cs, ci)
    assert np.array_equal(pos.cpu().numpy(), f["pos_wrapped"])
    g = D.compute_max_overlap(pos, rad, cs, cc, ci, lmd, n)
    assert np.float32(g) == f["max_overlap"]
    assert np.array_equal(lmd.cpu().numpy(), f["local_max_depth"])
    for s in range(2):
        D.project_overlaps(pos, rad, cs, cc, ci, n)
        assert np.array_equal(pos.cpu().numpy(), f[f"jacobi{s}"]), f"sweep {s}"
        Gr.rebuild_grid(pos, n, cc, cs, ci)


def test_pressure_matches_reference():
    f, m = load("pressure")
    n = m["n"]
    setup(n, DOMAIN_SIZE=1.0)
    from fos import dynamics as D
    rad = cuda(f["rad"])
    pos = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    dr = torch.zeros(n, dtype=torch.float32, device="cuda")
    ids, fsc = cuda(f["face_ids"]), cuda(f["fsc"])
    for s, (frame, nei) in enumerate(zip(m["frames"], m["max_nei"])):
        # each sweep starts from the reference's radii, so errors do not compound
        rad.copy_(cuda(f["rad"] if s == 0 else f[f"sweep{s - 1}_rad"]))
        mx, ch = D.equilibrate_pressure(n, frame, pos, rad, dr, ids, fsc, m["k"], m["P_exp"],
                                        m["pair_cap"], nei, m["r_min"], m["r_max"])
        want = f[f"sweep{s}_rad"]
        got = rad.cpu().numpy()
        assert np.max(np.abs(got - want) / want) <= PRESSURE_RTOL, f"sweep {s}"
        assert abs(mx - f[f"sweep{s}_ret"][0]) <= PRESSURE_RTOL * max(mx, 1e-30) + 1e-9
        assert abs(ch - f[f"sweep{s}_ret"][1]) <= 2


def test_controller_matches_reference():
    f, m = load("controller")
    n = m["n"]
    setup(n, DOMAIN_SIZE=1.0)
    from fos import dynamics as D
    rad, fsc, ema, lmd = cuda(f["rad"]), cuda(f["fsc"]), cuda(f["ema"]), cuda(f["lmd"])
    rt = torch.zeros(n, dtype=torch.float32, device="cuda")
    D.set_fsc_targets(rad, rt, fsc, ema, n, m["f_low"], m["f_high"], m["growth_pct"],
                      m["r_min"], m["r_max"])
    assert np.array_equal(rt.cpu().numpy(), f["rad_target"])
    g, s, i, md, mxd = D.compute_controller_stats(rad, rt, ema, n, m["f_low"], m["f_high"])
    want = f["controller_stats"]
    assert (g, s, i) == tuple(int(x) for x in want[:3])
    assert abs(md - want[3]) <= 1e-6 * abs(want[3]) + 1e-12
    assert np.float32(mxd) == np.float32(want[4])
    for mode in (0, 1, 2):
        r = cuda(f["rad"])
        D.nudge_radii_adaptive_ema(r, rt, lmd, n, m["alpha"], m["max_step_pct"], m["r_min"],
                                   m["r_max"], m["back_global"], mode)
        assert np.array_equal(r.cpu().numpy(), f[f"nudge_mode{mode}"]), f"mode {mode}"


def test_brownian_matches_reference():
    f, m = load("brownian")
    n = m["n"]
    setup(n, DOMAIN_SIZE=m["domain"], SEED=m["seed"])
    from fos import dynamics as D
    D._brownian_calls = 0
    pos = cuda(f["pos"])
    for fr in (0, 1):
        D.apply_brownian_motion(pos, n, m["strength"], m["domain"])
        assert np.array_equal(pos.cpu().numpy(), f[f"frame{fr}_pos"]), f"frame {fr}"


def test_ou_jitter_matches_reference():
    f, m = load("ou_jitter")
    n = m["n"]
    setup(n, DOMAIN_SIZE=1.0, SEED=m["seed"], JITTER_ENABLED=True, JITTER_RMS=m["rms"],
          JITTER_TAU=m["tau"], MAX_DRIFT_FRACTION=m["max_drift"], GAP_FRACTION=m["gap"])
    from fos import dynamics as D
    D._jitter_calls = 0
    pos, rad = cuda(f["pos"]), cuda(f["rad"])
    vj = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    D.init_jitter_velocities(vj, n)
    mr = torch.zeros(1, dtype=torch.float32, device="cuda")
    for fr in range(3):
        mr.fill_(float(f[f"frame{fr}_mean_radius"]))
        D.apply_brownian(vj, rad, mr, n, m["dt"])
        D.integrate_jitter(pos, vj, n, m["dt"])
        assert np.array_equal(vj.cpu().numpy(), f[f"frame{fr}_v_jit"]), f"frame {fr}: v_jit"
        assert np.array_equal(pos.cpu().numpy(), f[f"frame{fr}_pos"]), f"frame {fr}: pos"


def test_dirty_tiles_match_reference():
    f, m = load("dirty_tiles")
    n, R = m["n"], m["R"]
    jfa = setup(n, R, DOMAIN_SIZE=m["L"])
    jfa.set_resolution(R)
    jfa.update_tile_cache(cuda(f["pos_prev"]), cuda(f["rad_prev"]), n)
    jfa.clear_dirty_tiles()
    jfa.mark_dirty_tiles(cuda(f["pos"]), cuda(f["rad"]), n)
    assert np.array_equal(jfa.tile_dirty.to_numpy(), f["dirty"])
    assert jfa.count_dirty_tiles() == f["count"]
