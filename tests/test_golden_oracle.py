"""The CPU oracle against golden fixtures of the reference's own execution.

tests/golden/*.npz hold what the unmodified reference modules (jfa.py,
grid.py, dynamics.py) computed on small seeded inputs, executed serially
under the Taichi stand-in (tests/golden/make_golden.py).  Every stage of the
oracle must reproduce them bit for bit: owner labels, filtered labels, face
rows in slot order, neighbour lists, FSC, the EMA and the hysteresis scores
over consecutive runs, the pass count and per-pass changes (early exit
included), cell lists, PBD sweeps, overlap depths, pressure sweeps (the same
libm powf on both sides), the controller, Brownian and OU jitter, and the
dirty tiles.
"""
import ctypes as C
import glob
import json
import os
from dataclasses import dataclass

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    return {k: z[k] for k in z.files}, json.loads(str(z["meta"]))


@dataclass
class GridParams(O.OracleParams):
    grid_res: int = 3

    @property
    def G(self) -> int:
        return self.grid_res


def test_every_fixture_is_checked():
    names = {os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "*.npz"))}
    assert names == set(JFA_CASES) | {"grid_g3", "grid_g5", "pbd_g4", "pressure", "controller",
                                      "brownian", "ou_jitter", "dirty_tiles"}


JFA_CASES = ["jfa_r16_hysteresis", "jfa_r24_ties_early_exit", "jfa_r16_domain0189",
             "jfa_r24_overflow", "jfa_r36_crowded", "jfa_r16_crowded"]


@pytest.mark.parametrize("case", JFA_CASES)
def test_jfa_runs_match_reference(case):
    f, m = load(case)
    n, R = m["n"], m["R"]
    p = O.OracleParams(n=n, L=m["L"], R=R, early_exit=m["early_exit"],
                       th_delta=m.get("th_delta", 0.006), t_add=m.get("t_add", 0.15),
                       t_drop=m.get("t_drop", 0.10))
    prev = np.zeros((n, 32), np.float32)
    ema = np.zeros(n, np.float32)
    for k in range(m["runs"]):
        # the reference ran at the recorded resolution (set_resolution clamps)
        assert f[f"run{k}_labels"].size == R ** 3
        pos, rad = f[f"run{k}_pos"], f[f"run{k}_rad"]
        lab, changes, passes = O.jfa_labels(pos, rad, p)
        assert passes == f[f"run{k}_stat_num_passes"]
        assert np.array_equal(changes, f[f"run{k}_stat_changes"])
        assert np.array_equal(lab, f[f"run{k}_labels"]), f"run {k}: labels"
        filt = O.majority_filter(lab, R)
        assert np.array_equal(filt, f[f"run{k}_filtered"]), f"run {k}: filtered labels"
        ids, cnt = O.accumulate_faces(filt, R, n)
        assert np.array_equal(ids, f[f"run{k}_face_ids"]), f"run {k}: face_ids"
        assert np.array_equal(cnt, f[f"run{k}_face_counts"]), f"run {k}: face_counts"
        nl, used, fsc = O.finalize(rad, ids, cnt, prev, p)
        O.fsc_ema(fsc, ema, p.ema_alpha)
        assert np.array_equal(nl, f[f"run{k}_neighbor_list"]), f"run {k}: neighbor_list"
        assert np.array_equal(used, f[f"run{k}_neighbor_used_count"])
        assert np.array_equal(fsc, f[f"run{k}_fsc"]), f"run {k}: fsc"
        assert np.array_equal(prev, f[f"run{k}_prev_scores"]), f"run {k}: prev scores"
        assert np.array_equal(ema, f[f"run{k}_fsc_ema"]), f"run {k}: fsc_ema"
        assert used.sum() == f[f"run{k}_stat_p_dir"]
        assert (used >= 32).sum() == f[f"run{k}_stat_overflow_count"]
        assert fsc.min() == f[f"run{k}_stat_min_fsc"] and fsc.max() == f[f"run{k}_stat_max_fsc"]
        assert abs(fsc.mean() - f[f"run{k}_stat_mean_fsc"]) <= 1e-5 * max(1.0, fsc.mean())


def test_fixture_cases_reach_their_edges():
    """The fixtures hold the situations they were built for."""
    f, _ = load("jfa_r24_overflow")
    for k in range(2):
        assert (f[f"run{k}_face_ids"][0] >= 0).all()          # face row 0 full
        assert f[f"run{k}_stat_overflow_count"] > 0           # a neighbour list full
    f, m = load("jfa_r24_ties_early_exit")
    assert m["early_exit"] and f["run0_stat_early_exit"] == 1
    assert f["run0_stat_num_passes"] < 6                      # stopped before the last pass
    f, _ = load("jfa_r16_hysteresis")
    assert not np.array_equal(f["run1_prev_scores"], f["run2_prev_scores"])


@pytest.mark.parametrize("case", ["grid_g3", "grid_g5"])
def test_grid_build_matches_reference(case):
    f, m = load(case)
    p = GridParams(n=m["n"], L=m["L"], grid_res=m["G"])
    pos = f["pos"].copy()
    cc, cs, ci = O.grid_build(pos, p)
    assert np.array_equal(pos, f["pos_wrapped"])
    assert np.array_equal(cc, f["cell_count"])
    assert np.array_equal(cs, f["cell_start"])
    assert np.array_equal(ci, f["cell_indices"])


def test_pbd_and_max_overlap_match_reference():
    f, m = load("pbd_g4")
    p = GridParams(n=m["n"], L=m["L"], grid_res=m["G"])
    rad = f["rad"]
    pos = f["pos"].copy()
    grid = O.grid_build(pos, p)
    assert np.array_equal(pos, f["pos_wrapped"])
    g, lm = O.max_overlap(pos, rad, grid, p)
    assert np.float32(g) == f["max_overlap"]
    assert np.array_equal(lm, f["local_max_depth"])
    for s in range(2):
        pos = O.pbd(pos, rad, grid, p)
        assert np.array_equal(pos, f[f"jacobi{s}"]), f"sweep {s}"
        grid = O.grid_build(pos, p)


def test_pressure_matches_reference():
    f, m = load("pressure")
    rad = f["rad"].copy()
    for s, (frame, nei) in enumerate(zip(m["frames"], m["max_nei"])):
        p = O.OracleParams(n=m["n"], k=m["k"], P=m["P_exp"], pair_cap=m["pair_cap"],
                           max_nei=nei, r_min=m["r_min"], r_max=m["r_max"])
        mx, ch, dr = O.pressure(rad, f["face_ids"], f["fsc"], frame, p)
        assert np.array_equal(dr, f[f"sweep{s}_delta_r"]), f"sweep {s}: delta_r"
        assert np.array_equal(rad, f[f"sweep{s}_rad"]), f"sweep {s}: radii"
        assert np.float32(mx) == np.float32(f[f"sweep{s}_ret"][0])
        assert ch == f[f"sweep{s}_ret"][1]


def test_controller_matches_reference():
    f, m = load("controller")
    n = m["n"]
    p = O.OracleParams(n=n, f_low=m["f_low"], f_high=m["f_high"], growth=m["growth_pct"],
                       r_min=m["r_min"], r_max=m["r_max"])
    rt = np.empty(n, np.float32)
    O.set_targets(f["rad"], rt, f["fsc"], f["ema"], p)
    assert np.array_equal(rt, f["rad_target"])
    f32 = O._f32
    for mode in (0, 1, 2):
        rad = f["rad"].copy()
        O.lib().orc_nudge(O._ptr(rad), O._ptr(rt), O._ptr(f["lmd"]), n, f32(m["alpha"]),
                          f32(m["max_step_pct"]), f32(m["r_min"]), f32(m["r_max"]),
                          f32(m["back_global"]), mode, f32(p.contact_tol))
        assert np.array_equal(rad, f[f"nudge_mode{mode}"]), f"mode {mode}"


def test_brownian_matches_reference():
    f, m = load("brownian")
    p = O.OracleParams(n=m["n"], brownian=m["strength"], L=m["domain"], seed=m["seed"])
    pos = f["pos"].copy()
    for fr in (0, 1):
        O.brownian(pos, p, fr)
        assert np.array_equal(pos, f[f"frame{fr}_pos"]), f"frame {fr}"


def test_ou_jitter_matches_reference():
    f, m = load("ou_jitter")
    n = m["n"]
    pos = f["pos"].copy()
    rad = f["rad"]
    vj = np.zeros((n, 3), np.float32)
    for fr in range(3):
        mr = f[f"frame{fr}_mean_radius"]
        O.lib().orc_ou_jitter(O._ptr(pos), O._ptr(vj), O._ptr(rad), n, C.c_float(mr),
                              O._f32(m["dt"]), float(m["rms"]), float(m["tau"]),
                              float(m["max_drift"]), float(m["gap"]), O._f32(1.0), O._f32(1.0),
                              int(m["seed"]), fr)
        assert np.array_equal(vj, f[f"frame{fr}_v_jit"]), f"frame {fr}: v_jit"
        assert np.array_equal(pos, f[f"frame{fr}_pos"]), f"frame {fr}: positions"


def test_mean_radius_matches_run_py():
    """run.py takes numpy's float32 mean (run.py:860-861); the oracle's exact
    fixed-point mean rounds once.  They agree to one float32 ulp."""
    f, m = load("ou_jitter")
    mr = f["frame0_mean_radius"]
    assert abs(O.mean_radius(f["rad"], m["n"]) - mr) <= np.spacing(mr)


def test_dirty_tiles_match_reference():
    f, m = load("dirty_tiles")
    p = O.OracleParams(n=m["n"], L=m["L"], R=m["R"])
    T = m["tiles"]
    dirty = np.zeros((T, T, T), np.uint8)
    O.dirty_mark(f["pos"], f["rad"], f["pos_prev"], f["rad_prev"], dirty, p)
    assert np.array_equal(dirty, f["dirty"])
    assert O.dirty_count(dirty, m["R"]) == f["count"]
