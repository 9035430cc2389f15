"""Golden fixtures from the reference's own code.

TEST INFRASTRUCTURE.  Runs the UNMODIFIED reference modules (config.py,
grid.py, dynamics.py, jfa.py of Fabric-of-Space-Taichi-JFA) under the serial
Taichi stand-in in ``tests/golden/standin/`` on small seeded inputs, and writes
one ``tests/golden/<case>.npz`` per case: the inputs, the reference's outputs
and a JSON ``meta`` record (the configuration overrides and the calls made).

The reference cannot travel to the GPU hosts and Taichi cannot be installed,
so the fixtures are committed; ``tests/test_golden_oracle.py`` checks the CPU
oracle against them and ``tests/test_gpu_golden.py`` checks the CUDA path.

Configuration: ``config.py`` is imported as it is, then the module globals
that a case changes (domain size, cell size, the JFA resolution bounds that
``set_resolution`` clamps to, early exit) are set before ``grid``,
``dynamics`` and ``jfa`` import them.  Derived values are recomputed with
config.py's own formulas: HALF_L and INV_L (config.py:213-214) and GRID_RES
(config.py:317).  Each case loads the modules fresh, in its own process.

Calls follow run.py: ``rebuild_grid`` (run.py:476-504) is clear_grid,
count_particles_per_cell, prefix_sum, copy_cell_pointers, scatter_particles;
JFA runs go through ``jfa.run_jfa`` (jfa.py:1056-1197) with the reference's
own pass schedule.

``ti.random()`` draws come from Philox-4x32-10 with counter
(i, frame, stream, 0) and key = seed, u = (x >> 8) * 2^-24, taken in the order
the reference's kernel asks for them (particle by particle, axis by axis).
Both sides of every comparison therefore see identical jitter.

Usage:  python tests/golden/make_golden.py [--reference DIR] [--jobs N] [case ...]
"""
from __future__ import annotations

import argparse
import contextlib
import importlib
import io
import json
import math
import multiprocessing as mp
import os
import sys
import time
from types import SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
STANDIN = os.path.join(HERE, "standin")
DEFAULT_REFERENCE = "/root/reference"

BROW = 0x42524F57   # 'BROW': the Brownian stream word
OUJT = 0x4F554A54   # 'OUJT': the OU-jitter stream word


# ------------------------------------------------------------------ loading
def load_reference(ref_dir: str, **over):
    """Fresh import of the reference modules with config overrides applied."""
    for p in (STANDIN, ref_dir):
        if p not in sys.path:
            sys.path.insert(0, p)
    for m in ("config", "grid", "dynamics", "jfa", "topology"):
        sys.modules.pop(m, None)
    import taichi as ti
    quiet = io.StringIO()
    with contextlib.redirect_stdout(quiet):
        config = importlib.import_module("config")
    L = over.pop("DOMAIN_SIZE", config.DOMAIN_SIZE)
    config.DOMAIN_SIZE = L
    config.HALF_L = 0.5 * L            # config.py:213
    config.INV_L = 1.0 / L             # config.py:214
    cs = over.pop("CELL_SIZE", None)
    if cs is not None:
        config.CELL_SIZE = cs
        config.GRID_RES = max(3, int(math.ceil(L / cs)))   # config.py:317
    config.JFA_RES_MIN = over.pop("JFA_RES_MIN", 8)
    config.JFA_RES_MAX = over.pop("JFA_RES_MAX", 32)
    for k, v in over.items():
        if not hasattr(config, k):
            raise KeyError(f"config has no {k}")
        setattr(config, k, v)
    with contextlib.redirect_stdout(quiet):
        grid = importlib.import_module("grid")
        dynamics = importlib.import_module("dynamics")
        jfa = importlib.import_module("jfa")
    jfa.init_jfa()
    return SimpleNamespace(ti=ti, config=config, grid=grid, dynamics=dynamics, jfa=jfa)


def particle_fields(ref, pos: np.ndarray, rad: np.ndarray):
    ti = ref.ti
    n = len(rad)
    p = ti.Vector.field(3, dtype=ti.f32, shape=n)
    r = ti.field(dtype=ti.f32, shape=n)
    p.from_numpy(np.ascontiguousarray(pos, np.float32))
    r.from_numpy(np.ascontiguousarray(rad, np.float32))
    return p, r


def grid_fields(ref, n: int):
    ti = ref.ti
    G3 = ref.config.GRID_RES ** 3
    return SimpleNamespace(count=ti.field(dtype=ti.i32, shape=G3),
                           start=ti.field(dtype=ti.i32, shape=G3),
                           write=ti.field(dtype=ti.i32, shape=G3),
                           indices=ti.field(dtype=ti.i32, shape=n))


def rebuild_grid(ref, g, pos, n: int):
    """run.py:476-504"""
    G = ref.grid
    G.clear_grid(g.count)
    G.count_particles_per_cell(pos, g.count, n)
    G.prefix_sum(g.count, g.start)
    G.copy_cell_pointers(g.start, g.write)
    G.scatter_particles(pos, g.write, g.indices, n)


def philox_draws(n: int, frame: int, stream: int, seed: int) -> np.ndarray:
    """u[i, d] for d in 0..2: (x_d >> 8) * 2^-24 of Philox-4x32-10."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    u = np.empty((n, 3), np.float32)
    for i in range(n):
        w = O.philox((i, frame, stream, 0), (seed & 0xFFFFFFFF, seed >> 32))
        for d in range(3):
            u[i, d] = np.float32(int(w[d]) >> 8) * np.float32(2.0 ** -24)
    return u


def feed_random(ref, draws: np.ndarray):
    it = iter(draws.reshape(-1).tolist())

    def source(dtype):
        return np.float32(next(it))
    ref.ti.set_random_source(source)


def jfa_state(ref, n: int) -> dict:
    j = ref.jfa
    R = j.JFA_RES
    return {
        "labels": j.jfa_grid.to_numpy()[:R, :R, :R, 0].astype(np.int32).reshape(-1),
        "filtered": j.label_filtered.to_numpy()[:R, :R, :R].reshape(-1).copy(),
        "face_ids": j.face_ids.to_numpy()[:n].copy(),
        "face_counts": j.face_counts.to_numpy()[:n].copy(),
        "neighbor_list": j.neighbor_list.to_numpy()[:n].copy(),
        "neighbor_used_count": j.neighbor_used_count.to_numpy()[:n].copy(),
        "fsc": j.fsc.to_numpy()[:n].copy(),
        "fsc_ema": j.fsc_ema.to_numpy()[:n].copy(),
        "prev_scores": j.neighbor_prev_scores.to_numpy()[:n].copy(),
    }


def stats_arrays(stats: dict, V: int) -> dict:
    return {
        "num_passes": np.int32(stats["num_passes"]),
        "early_exit": np.int32(bool(stats["early_exit"])),
        "changes": np.array([round(d * V) for d in stats["delta_history"]], np.int64),
        "p_dir": np.int64(stats["p_dir"]),
        "overflow_count": np.int64(stats["overflow_count"]),
        "min_fsc": np.int64(stats["min_fsc"]),
        "max_fsc": np.int64(stats["max_fsc"]),
        "mean_fsc": np.float64(stats["mean_fsc"]),
        "mean_fsc_ema": np.float64(stats["mean_fsc_ema"]),
        "mean_score": np.float64(stats["mean_score"]),
        "std_score": np.float64(stats["std_score"]),
    }


# -------------------------------------------------------------------- cases
def _jfa_runs(ref, pos0, rad0, runs: int, rng, move: float, grow: float):
    """run_jfa `runs` times, moving and rescaling the particles in between."""
    n = len(rad0)
    out = {}
    pos, rad = pos0.copy(), rad0.copy()
    V = ref.jfa.JFA_RES ** 3
    for k in range(runs):
        pf, rf = particle_fields(ref, pos, rad)
        fsc, stats = ref.jfa.run_jfa(pf, rf, n)
        st = jfa_state(ref, n)
        assert np.array_equal(st["fsc"], fsc)
        val = ref.jfa.validate_jfa(n)
        out[f"run{k}_pos"] = pos.copy()
        out[f"run{k}_rad"] = rad.copy()
        for key, v in st.items():
            out[f"run{k}_{key}"] = v
        for key, v in stats_arrays(stats, V).items():
            out[f"run{k}_stat_{key}"] = v
        out[f"run{k}_validate"] = np.array([int(bool(val["passed"])), val["asymmetric_pairs"],
                                            val["overflow_count"], val["self_loops"]], np.int64)
        pos = (pos + rng.uniform(-move, move, pos.shape)).astype(np.float32)
        rad = (rad * rng.uniform(1.0 - grow, 1.0 + grow, n)).astype(np.float32)
    return out


def case_jfa_r16_hysteresis(ref_dir):
    """R = 16 (5 passes), 40 cells, three runs with moves in between, so that
    neighbor_prev_scores carries the hysteresis from run to run."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0, JFA_EARLY_EXIT_ENABLED=False)
    ref.jfa.set_resolution(16)
    rng = np.random.default_rng(1601)
    n = 40
    pos = (rng.random((n, 3), dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    rad = rng.uniform(0.05, 0.09, n).astype(np.float32)
    out = _jfa_runs(ref, pos, rad, 3, rng, 0.02, 0.15)
    meta = dict(L=1.0, R=16, n=n, runs=3, early_exit=False, calls="jfa.run_jfa x3")
    return out, meta


def case_jfa_r24_ties_early_exit(ref_dir):
    """R = 24 (not a power of two: steps 12, 6, 3, 1, 1, 1), early exit on with
    TH_PASS_DELTA = 0.02 so that it stops a pass early, coincident seeds with different radii, an exact
    duplicate (pos and radius: a tie the first index wins), and positions
    outside [-L/2, L/2) that the voxel mapping wraps."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0, JFA_EARLY_EXIT_ENABLED=True,
                         TH_PASS_DELTA=0.02)
    ref.jfa.set_resolution(24)
    rng = np.random.default_rng(2402)
    n = 48
    pos = (rng.random((n, 3), dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    rad = rng.uniform(0.04, 0.07, n).astype(np.float32)
    pos[5] = pos[3]                      # same voxel, different radius
    pos[7], rad[7] = pos[2], rad[2]      # exact duplicate: a tie
    pos[11] = pos[11] + np.float32(1.0)  # unwrapped copies of in-box positions
    pos[12] = pos[12] - np.float32(1.0)
    pos[13] = np.array([-0.5, 0.0, 0.49999997], np.float32)
    out = _jfa_runs(ref, pos, rad, 2, rng, 0.015, 0.10)
    meta = dict(L=1.0, R=24, n=n, runs=2, early_exit=True, th_delta=0.02, min_passes=3,
                calls="jfa.run_jfa x2")
    return out, meta


def case_jfa_r16_domain0189(ref_dir):
    """The reference's own domain size L = 0.189 (config.py:21), so that
    HALF_L, INV_L and VOXEL_SIZE are not exact in f32."""
    L = 0.189
    ref = load_reference(ref_dir, DOMAIN_SIZE=L, JFA_EARLY_EXIT_ENABLED=False)
    ref.jfa.set_resolution(16)
    rng = np.random.default_rng(1603)
    n = 32
    pos = ((rng.random((n, 3), dtype=np.float32) - np.float32(0.5)) * np.float32(L)).astype(
        np.float32)
    rad = (rng.uniform(0.05, 0.09, n) * L).astype(np.float32)
    out = _jfa_runs(ref, pos, rad, 2, rng, 0.003, 0.1)
    meta = dict(L=L, R=16, n=n, runs=2, early_exit=False, calls="jfa.run_jfa x2")
    return out, meta


def case_jfa_r24_overflow(ref_dir):
    """Two large cells, each inside a shell of 40 small ones, with T_ADD and
    T_DROP lowered so that their small faces are accepted.  The large cell at
    index 0 meets more than 32 partners in its own face row, so
    accumulate_face_area drops the partners that find no free slot
    (jfa.py:746-762).  The large cell at the last index receives more than 32
    add_neighbor calls from other rows, so its list stops at MAX_NEIGHBORS
    (jfa.py:432-441)."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0, JFA_EARLY_EXIT_ENABLED=False)
    ref.jfa.T_ADD, ref.jfa.T_DROP = 0.02, 0.01
    ref.jfa.set_resolution(24)
    rng = np.random.default_rng(2404)
    m = 40
    parts_p, parts_r = [], []
    for centre in ((-0.25, 0.0, 0.0), (0.25, 0.0, 0.0)):
        v = rng.normal(size=(m, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        parts_p.append((np.array(centre) + v * 0.21).astype(np.float32))
        parts_r.append(rng.uniform(0.025, 0.035, m).astype(np.float32))
    pos = np.concatenate([np.array([[-0.25, 0.0, 0.0]], np.float32), *parts_p,
                          np.array([[0.25, 0.0, 0.0]], np.float32)]).astype(np.float32)
    rad = np.concatenate([[0.18], *parts_r, [0.18]]).astype(np.float32)
    out = _jfa_runs(ref, pos, rad, 2, rng, 0.005, 0.05)
    meta = dict(L=1.0, R=24, n=len(rad), runs=2, early_exit=False, t_add=0.02, t_drop=0.01,
                calls="jfa.run_jfa x2")
    return out, meta


def case_jfa_r36_crowded(ref_dir):
    """R = 36: not a power of two and not a multiple of 8 (7 passes: steps 18,
    9, 4, 2, 1, 1, 1), with 150 small cells of about 300 voxels each, so that
    many distinct face pairs meet in every region of the grid."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0, JFA_EARLY_EXIT_ENABLED=False, JFA_RES_MAX=64)
    ref.jfa.set_resolution(36)
    assert ref.jfa.JFA_RES == 36  # not clamped by set_resolution
    rng = np.random.default_rng(3606)
    n = 150
    pos = (rng.random((n, 3), dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    rad = rng.uniform(0.02, 0.05, n).astype(np.float32)
    out = _jfa_runs(ref, pos, rad, 2, rng, 0.01, 0.10)
    meta = dict(L=1.0, R=36, n=n, runs=2, early_exit=False, calls="jfa.run_jfa x2")
    return out, meta


def case_jfa_r16_crowded(ref_dir):
    """R = 16 with 400 seeds (about ten voxels a cell; 19 seeds own no
    voxel), so that most voxel faces separate two cells and a face row holds
    up to 26 partners."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0, JFA_EARLY_EXIT_ENABLED=False)
    ref.jfa.set_resolution(16)
    assert ref.jfa.JFA_RES == 16
    rng = np.random.default_rng(1616)
    n = 400
    pos = (rng.random((n, 3), dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    rad = rng.uniform(0.01, 0.03, n).astype(np.float32)
    out = _jfa_runs(ref, pos, rad, 2, rng, 0.01, 0.10)
    meta = dict(L=1.0, R=16, n=n, runs=2, early_exit=False, calls="jfa.run_jfa x2")
    return out, meta


def _edge_positions(G: int, L: float, rng, n: int) -> np.ndarray:
    f = np.float32
    pos = (rng.random((n, 3), dtype=np.float32) - f(0.5)).astype(np.float32)
    cell = L / G
    edges = [f(-0.5 * L), f(-0.5 * L + cell), f(0.0), f(0.5 * L - cell), f(0.49999997 * L),
             f(0.5 * L), f(0.75 * L), f(-0.6 * L), f(1.3 * L), f(-1.2 * L)]
    k = 0
    for e in edges:
        for d in range(3):
            pos[k, d] = e
            k += 1
            if k >= n:
                return pos
    return pos


def _grid_case(ref_dir, G: int, n: int, seed: int):
    L = 1.0
    ref = load_reference(ref_dir, DOMAIN_SIZE=L, CELL_SIZE=L / G)
    assert ref.config.GRID_RES == G
    rng = np.random.default_rng(seed)
    pos = _edge_positions(G, L, rng, n)
    rad = rng.uniform(0.01, 0.02, n).astype(np.float32)
    pf, rf = particle_fields(ref, pos, rad)
    g = grid_fields(ref, n)
    rebuild_grid(ref, g, pf, n)
    out = dict(pos=pos, rad=rad, cell_count=g.count.to_numpy(), cell_start=g.start.to_numpy(),
               cell_indices=g.indices.to_numpy(), pos_wrapped=pf.to_numpy())
    meta = dict(L=L, G=G, n=n, calls="rebuild_grid (run.py:476-504)")
    return out, meta


def case_grid_g3(ref_dir):
    """GRID_RES = 3 (the minimum), positions on cell faces and outside the box."""
    return _grid_case(ref_dir, 3, 40, 303)


def case_grid_g5(ref_dir):
    """GRID_RES = 5 (odd), positions on cell faces and outside the box."""
    return _grid_case(ref_dir, 5, 64, 505)


def _pbd_jacobi(ref, pos: np.ndarray, rad: np.ndarray) -> np.ndarray:
    """One Jacobi sweep of the reference's project_overlaps.

    The serial kernel updates index 0 before it writes anything that index 0
    reads.  So particle i's Jacobi update is what the kernel computes for
    index 0 when i is moved to the front.  The other particles keep their
    relative order, so every cell list visits them in the same order."""
    n = len(rad)
    out = np.empty_like(pos)
    for i in range(n):
        perm = np.array([i] + [j for j in range(n) if j != i])
        pf, rf = particle_fields(ref, pos[perm], rad[perm])
        g = grid_fields(ref, n)
        rebuild_grid(ref, g, pf, n)
        ref.dynamics.project_overlaps(pf, rf, g.start, g.count, g.indices, n)
        out[i] = pf.to_numpy()[0]
    return out


def case_pbd_g4(ref_dir):
    """Two PBD sweeps with a grid rebuild before each (run.py:829-846), as
    Jacobi sweeps of the reference's own kernel, then the serial
    (Gauss-Seidel) sweep the kernel gives as written, and the local and
    global maximum overlap (dynamics.py:304-372)."""
    L, G = 1.0, 4
    ref = load_reference(ref_dir, DOMAIN_SIZE=L, CELL_SIZE=L / G)
    rng = np.random.default_rng(404)
    n = 40
    pos = _edge_positions(G, L, rng, n)
    rad = rng.uniform(0.08, 0.125, n).astype(np.float32)
    out = dict(pos=pos.copy(), rad=rad)
    # wrap once through a rebuild, as the frame's first grid build does
    pf, rf = particle_fields(ref, pos, rad)
    g = grid_fields(ref, n)
    rebuild_grid(ref, g, pf, n)
    cur = pf.to_numpy()
    out["pos_wrapped"] = cur.copy()
    lmd = ref.ti.field(dtype=ref.ti.f32, shape=n)
    omax = ref.dynamics.compute_max_overlap(pf, rf, g.start, g.count, g.indices, lmd, n)
    out["max_overlap"] = np.float32(omax)
    out["local_max_depth"] = lmd.to_numpy()
    for s in range(2):
        cur = _pbd_jacobi(ref, cur, rad)
        out[f"jacobi{s}"] = cur.copy()
    pf, rf = particle_fields(ref, out["pos_wrapped"], rad)
    g = grid_fields(ref, n)
    rebuild_grid(ref, g, pf, n)
    ref.dynamics.project_overlaps(pf, rf, g.start, g.count, g.indices, n)
    out["gauss_seidel0"] = pf.to_numpy()
    meta = dict(L=L, G=G, n=n, calls="rebuild_grid + compute_max_overlap; 2 x (rebuild_grid + "
                "project_overlaps) as Jacobi sweeps; one serial project_overlaps")
    return out, meta


def case_pressure(ref_dir):
    """equilibrate_pressure (dynamics.py:1454-1557) over six frames on
    hand-made face rows: empty rows, rows longer than max_nei, entries of -1,
    entries >= n and self entries (all skipped), radii at both clamps."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0)
    ti = ref.ti
    rng = np.random.default_rng(7007)
    n = 50
    rad = rng.uniform(0.02, 0.05, n).astype(np.float32)
    rad[0], rad[1] = np.float32(0.0201), np.float32(0.0499)
    fsc = rng.integers(0, 21, n).astype(np.int32)
    fsc[2], fsc[3] = 0, 32
    ids = rng.integers(-1, n + 3, (n, 32)).astype(np.int32)
    ids[4, :5] = 4
    pos = np.zeros((n, 3), np.float32)
    pf, rf = particle_fields(ref, pos, rad)
    fid = ti.field(dtype=ti.i32, shape=(n, 32))
    ff = ti.field(dtype=ti.i32, shape=n)
    dr = ti.field(dtype=ti.f32, shape=n)
    fid.from_numpy(ids)
    ff.from_numpy(fsc)
    out = dict(rad=rad.copy(), face_ids=ids, fsc=fsc)
    params = dict(k=0.10, P_exp=3.0, pair_cap=0.02, r_min=0.02, r_max=0.05)
    frames = [0, 1, 2, 17, 123456, 2147483]
    nei = [10, 10, 3, 10, 32, 10]
    for s, (fr, mn) in enumerate(zip(frames, nei)):
        mx, ch = ref.dynamics.equilibrate_pressure(n, fr, pf, rf, dr, fid, ff, params["k"],
                                                   params["P_exp"], params["pair_cap"], mn,
                                                   params["r_min"], params["r_max"])
        out[f"sweep{s}_rad"] = rf.to_numpy()
        out[f"sweep{s}_delta_r"] = dr.to_numpy()
        out[f"sweep{s}_ret"] = np.array([mx, ch], np.float64)
    meta = dict(n=n, frames=frames, max_nei=nei, **params,
                calls="dynamics.equilibrate_pressure per frame")
    return out, meta


def case_controller(ref_dir):
    """set_fsc_targets (dynamics.py:1242-1320), compute_controller_stats and
    nudge_radii_adaptive_ema (dynamics.py:1366-1427) in modes off, global and
    local, with FSC values on every branch and radii at both clamps."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0)
    ti = ref.ti
    rng = np.random.default_rng(8008)
    n = 64
    f_low, f_high = 10, 16
    rad = rng.uniform(0.02, 0.05, n).astype(np.float32)
    rad[0], rad[1] = np.float32(0.05), np.float32(0.02)
    ema = rng.uniform(6.0, 20.0, n).astype(np.float32)
    fsc = rng.integers(5, 21, n).astype(np.int32)
    pts = [0.0, 8.0, 8.999, 9.0, 9.5, 9.99, 10.0, 12.99, 13.0, 13.01, 16.0, 16.01, 16.5,
           17.0, 17.01, 25.0]
    ema[:len(pts)] = np.array(pts, np.float32)
    ema[0] = 0.0
    fsc[0] = 7
    lmd = rng.uniform(0.0, 0.05, n).astype(np.float32)
    lmd[2], lmd[3] = np.float32(0.035), np.float32(0.0)
    rt = ti.field(dtype=ti.f32, shape=n)
    fields = {}
    for name, arr, dt in (("rad", rad, ti.f32), ("fsc", fsc, ti.i32), ("ema", ema, ti.f32),
                          ("lmd", lmd, ti.f32)):
        fields[name] = ti.field(dtype=dt, shape=n)
        fields[name].from_numpy(arr)
    D = ref.dynamics
    D.set_fsc_targets(fields["rad"], rt, fields["fsc"], fields["ema"], n, f_low, f_high, 0.10,
                      0.02, 0.05)
    out = dict(rad=rad, fsc=fsc, ema=ema, lmd=lmd, rad_target=rt.to_numpy())
    cs = D.compute_controller_stats(fields["rad"], rt, fields["ema"], n, f_low, f_high)
    out["controller_stats"] = np.array(cs, np.float64)
    alpha = 1.0 - (0.05 ** (1.0 / max(1, 15)))     # run.py:440-452, ADJUSTMENT_FRAMES = 15
    back_global = 0.6
    for mode in (0, 1, 2):
        fields["rad"].from_numpy(rad)
        D.nudge_radii_adaptive_ema(fields["rad"], rt, fields["lmd"], n, alpha, 0.12, 0.02, 0.05,
                                   back_global, mode)
        out[f"nudge_mode{mode}"] = fields["rad"].to_numpy()
    meta = dict(n=n, f_low=f_low, f_high=f_high, growth_pct=0.10, r_min=0.02, r_max=0.05,
                alpha=alpha, max_step_pct=0.12, back_global=back_global,
                calls="set_fsc_targets, compute_controller_stats, nudge_radii_adaptive_ema x3")
    return out, meta


def case_brownian(ref_dir):
    """apply_brownian_motion (dynamics.py:1596-1634) over two frames with a
    large strength, particles near both faces so that both wrap branches run."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0)
    rng = np.random.default_rng(9009)
    n = 64
    seed = 77
    strength, domain = 0.02, 1.0
    pos = (rng.random((n, 3), dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    pos[:8] = np.float32(0.495)
    pos[8:16] = np.float32(-0.495)
    pos[16] = np.float32(-0.5)
    rad = np.full(n, 0.01, np.float32)
    pf, _ = particle_fields(ref, pos, rad)
    out = dict(pos=pos.copy(), seed=np.uint64(seed))
    for fr in (0, 1):
        feed_random(ref, philox_draws(n, fr, BROW, seed))
        ref.dynamics.apply_brownian_motion(pf, n, strength, domain)
        out[f"frame{fr}_pos"] = pf.to_numpy()
    meta = dict(n=n, seed=seed, strength=strength, domain=domain, stream="BROW",
                calls="apply_brownian_motion, frames 0 and 1")
    return out, meta


def case_ou_jitter(ref_dir):
    """apply_brownian + integrate_jitter (dynamics.py:607-660) over three
    frames, with run.py's mean radius (run.py:857-861); some particles hit
    the drift cap."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0, JITTER_ENABLED=True)
    ti = ref.ti
    rng = np.random.default_rng(1010)
    n = 48
    seed = 5
    dt = ref.config.DT
    pos = (rng.random((n, 3), dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    rad = rng.uniform(0.005, 0.05, n).astype(np.float32)
    rad[:6] = np.float32(1e-4)              # tiny cells: the drift cap binds
    pf, rf = particle_fields(ref, pos, rad)
    vj = ti.Vector.field(3, dtype=ti.f32, shape=n)
    mean_radius = ti.field(dtype=ti.f32, shape=())
    ref.dynamics.init_jitter_velocities(vj, n)
    out = dict(pos=pos.copy(), rad=rad, seed=np.uint64(seed))
    for fr in range(3):
        rad_np = rf.to_numpy()[:n]
        mean_radius[None] = rad_np.mean()           # run.py:860-861
        out[f"frame{fr}_mean_radius"] = np.float32(mean_radius[None])
        feed_random(ref, philox_draws(n, fr, OUJT, seed))
        ref.dynamics.apply_brownian(vj, rf, mean_radius, n, dt)
        ref.dynamics.integrate_jitter(pf, vj, n, dt)
        out[f"frame{fr}_v_jit"] = vj.to_numpy()
        out[f"frame{fr}_pos"] = pf.to_numpy()
    c = ref.config
    meta = dict(n=n, seed=seed, dt=dt, rms=c.JITTER_RMS, tau=c.JITTER_TAU,
                max_drift=c.MAX_DRIFT_FRACTION, gap=c.GAP_FRACTION, stream="OUJT",
                calls="init_jitter_velocities; 3 x (mean radius, apply_brownian, "
                      "integrate_jitter)")
    return out, meta


def case_dirty_tiles(ref_dir):
    """mark_dirty_tiles / count_dirty_tiles / update_tile_cache
    (jfa.py:966-1049) at R = 128 (8 tiles of 16 voxels per axis): moves below
    and above the thresholds, radius changes, tile crossings and the periodic
    halo."""
    ref = load_reference(ref_dir, DOMAIN_SIZE=1.0, JFA_RES_MAX=128)
    ref.jfa.set_resolution(128)
    j = ref.jfa
    rng = np.random.default_rng(1111)
    n = 24
    vs = np.float32(1.0 / 128)
    pos0 = (rng.random((n, 3), dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    rad0 = rng.uniform(0.01, 0.03, n).astype(np.float32)
    pos_prev = pos0.copy()
    pos1 = pos0.copy()
    rad1 = rad0.copy()
    pos1[0, 0] += np.float32(0.49) * vs      # below the move threshold
    pos1[1, 1] += np.float32(0.51) * vs      # above it
    rad1[2] += np.float32(0.26) * vs         # radius change above its threshold
    rad1[3] += np.float32(0.24) * vs         # below it
    pos_prev[4] = np.array([0.2499, 0.0, 0.0], np.float32)
    pos1[4] = np.array([0.2501, 0.0, 0.0], np.float32)     # crosses a tile face by a hair
    pos1[5] = np.array([-0.49, -0.49, 0.49], np.float32)   # the halo wraps around the box
    pos_prev[5] = pos1[5] - np.float32(0.1)
    pf0, rf0 = particle_fields(ref, pos_prev, rad0)
    j.update_tile_cache(pf0, rf0, n)
    j.clear_dirty_tiles()
    pf1, rf1 = particle_fields(ref, pos1, rad1)
    j.mark_dirty_tiles(pf1, rf1, n)
    T = j.tiles_per_axis
    out = dict(pos_prev=pos_prev, rad_prev=rad0, pos=pos1, rad=rad1,
               dirty=j.tile_dirty.to_numpy()[:T, :T, :T].copy(),
               count=np.int32(j.count_dirty_tiles()))
    meta = dict(L=1.0, R=128, n=n, tiles=T, calls="update_tile_cache, clear_dirty_tiles, "
                "mark_dirty_tiles, count_dirty_tiles")
    return out, meta


CASES = {
    "jfa_r16_hysteresis": case_jfa_r16_hysteresis,
    "jfa_r24_ties_early_exit": case_jfa_r24_ties_early_exit,
    "jfa_r16_domain0189": case_jfa_r16_domain0189,
    "jfa_r24_overflow": case_jfa_r24_overflow,
    "jfa_r36_crowded": case_jfa_r36_crowded,
    "jfa_r16_crowded": case_jfa_r16_crowded,
    "grid_g3": case_grid_g3,
    "grid_g5": case_grid_g5,
    "pbd_g4": case_pbd_g4,
    "pressure": case_pressure,
    "controller": case_controller,
    "brownian": case_brownian,
    "ou_jitter": case_ou_jitter,
    "dirty_tiles": case_dirty_tiles,
}


def run_case(args):
    name, ref_dir = args
    t = time.time()
    out, meta = CASES[name](ref_dir)
    meta = dict(case=name, doc=" ".join(CASES[name].__doc__.split()), reference="unmodified "
                "config.py, grid.py, dynamics.py, jfa.py under tests/golden/standin", **meta)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=np.array(json.dumps(meta)),
                        **out)
    return name, time.time() - t


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--jobs", type=int, default=min(8, os.cpu_count() or 1))
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    names = a.cases or list(CASES)
    ctx = mp.get_context("spawn")
    with ctx.Pool(a.jobs) as pool:
        for name, dt in pool.imap_unordered(run_case, [(n, a.reference) for n in names]):
            print(f"{name}: {dt:.1f} s", flush=True)


if __name__ == "__main__":
    main()
