"""GPU parity of the JFA power diagram and FSC extraction against the oracle.

Bar: owner labels, filtered labels, face_ids/face_counts (slot order
included), fsc, neighbour lists, neighbour_prev_scores and fsc_ema are
bit-exact with the serial-semantics oracle on the same inputs.
"""
import numpy as np
import pytest
import torch

from fos import inputs
from fos.config import FosConfig
from fos.context import Context
from oracle import oracle as O

from helpers import oracle_params, wrapped

pytestmark = pytest.mark.gpu


def _ctx(foam, **over):
    cfg = FosConfig.for_foam(foam, **over)
    return cfg, Context(cfg, max_n=foam.n, max_res=cfg.JFA_RES)


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("name", ["small", "headline", "stress"])
def test_labels_and_fsc_bit_exact(name):
    foam = {"small": inputs.small, "headline": inputs.headline, "stress": inputs.stress}[name]()
    pos = wrapped(foam.pos)
    rad = foam.rad.copy()
    p = oracle_params(foam)
    lab, ch, done = O.jfa_labels(pos, rad, p)
    cfg, ctx = _ctx(foam)
    dpos, drad = _dev(pos), _dev(rad)
    ctx.jfa_run(dpos, drad, foam.n)
    torch.cuda.synchronize()
    st = ctx.jfa_stats(foam.n, drad)
    assert st["num_passes"] == done == p.passes
    assert st["label_changes"] == [int(c) for c in ch]
    glab = ctx.labels().cpu().numpy().reshape(-1)
    assert np.array_equal(glab, lab)
    filt = O.majority_filter(lab, p.R)
    assert np.array_equal(ctx.label_filtered().cpu().numpy().reshape(-1), filt)
    ids, cnt = O.accumulate_faces(filt, p.R, foam.n)
    assert np.array_equal(ctx.face_ids[: foam.n].cpu().numpy(), ids)
    assert np.array_equal(ctx.face_counts[: foam.n].cpu().numpy(), cnt)
    prev = np.zeros((foam.n, 32), np.float32)
    nl, used, fsc = O.finalize(rad, ids, cnt, prev, p)
    ema = np.zeros(foam.n, np.float32)
    O.fsc_ema(fsc, ema, p.ema_alpha)
    assert np.array_equal(ctx.fsc[: foam.n].cpu().numpy(), fsc)
    assert np.array_equal(ctx.neighbor_used_count[: foam.n].cpu().numpy(), used)
    assert np.array_equal(ctx.neighbor_list[: foam.n].cpu().numpy(), nl)
    assert np.array_equal(ctx.neighbor_prev_scores[: foam.n].cpu().numpy(), prev)
    assert np.array_equal(ctx.fsc_ema[: foam.n].cpu().numpy(), ema)
    v = ctx.validate(foam.n)
    assert v["self_loops"] == 0 and v["asymmetric_pairs"] == 0
    assert st["zero_fsc_count"] == int(np.sum(fsc == 0))


def test_hysteresis_history_over_several_runs():
    """neighbor_prev_scores carries across runs; moving particles change faces."""
    foam = inputs.small()
    p = oracle_params(foam)
    cfg, ctx = _ctx(foam)
    pos = wrapped(foam.pos)
    rad = foam.rad.copy()
    rng = np.random.default_rng(7)
    prev = np.zeros((foam.n, 32), np.float32)
    ema = np.zeros(foam.n, np.float32)
    for it in range(4):
        lab, _, _ = O.jfa_labels(pos, rad, p)
        ids, cnt = O.accumulate_faces(O.majority_filter(lab, p.R), p.R, foam.n)
        nl, used, fsc = O.finalize(rad, ids, cnt, prev, p)
        O.fsc_ema(fsc, ema, p.ema_alpha)
        ctx.jfa_run(_dev(pos), _dev(rad), foam.n)
        torch.cuda.synchronize()
        assert np.array_equal(ctx.fsc[: foam.n].cpu().numpy(), fsc), it
        assert np.array_equal(ctx.neighbor_list[: foam.n].cpu().numpy(), nl), it
        assert np.array_equal(ctx.neighbor_prev_scores[: foam.n].cpu().numpy(), prev), it
        assert np.array_equal(ctx.fsc_ema[: foam.n].cpu().numpy(), ema), it
        pos = wrapped(pos + rng.uniform(-0.004, 0.004, pos.shape).astype(np.float32))
        rad = (rad * rng.uniform(0.95, 1.05, rad.shape)).astype(np.float32)


@pytest.mark.parametrize("R,L", [(48, 1.0), (40, 0.189), (36, 1.0)])
def test_non_power_of_two_and_reference_box(R, L):
    """Non-power-of-two grids against the oracle; R = 36 (not a multiple of 8)
    also takes the untiled face kernel."""
    rng = np.random.default_rng(11)
    n = 300
    pos = wrapped(rng.uniform(0, L, (n, 3)).astype(np.float32), L)
    rad = rng.uniform(0.02 * L, 0.04 * L, n).astype(np.float32)
    p = O.OracleParams(n=n, R=R, L=L, r_max_cell=0.04 * L)
    lab, _, _ = O.jfa_labels(pos, rad, p)
    cfg = FosConfig(DOMAIN_SIZE=L, CELL_SIZE=0.08 * L, JFA_RES=R, JFA_RES_MIN=2, JFA_RES_MAX=R,
                    JFA_EARLY_EXIT_ENABLED=False, MAX_PARTICLES=n)
    ctx = Context(cfg, max_n=n, max_res=R)
    ctx.jfa_run(_dev(pos), _dev(rad), n)
    torch.cuda.synchronize()
    assert np.array_equal(ctx.labels().cpu().numpy().reshape(-1), lab)
    ids, cnt = O.accumulate_faces(O.majority_filter(lab, R), R, n)
    prev = np.zeros((n, 32), np.float32)
    nl, used, fsc = O.finalize(rad, ids, cnt, prev, p)
    assert np.array_equal(ctx.fsc[:n].cpu().numpy(), fsc)
    assert np.array_equal(ctx.neighbor_list[:n].cpu().numpy(), nl)


def test_face_tiles_with_crowded_pairs():
    """3,000 seeds on a 16^3 grid: cells are about one voxel, so a 4 x 8 x 8
    face tile meets more distinct pairs than its 256-slot shared table holds
    and the overflow goes to the global table directly.  face_ids,
    face_counts, fsc and the neighbour lists still equal the oracle's."""
    rng = np.random.default_rng(5)
    n, R, L = 3000, 16, 1.0
    pos = wrapped(rng.uniform(0, L, (n, 3)).astype(np.float32), L)
    rad = rng.uniform(0.002, 0.004, n).astype(np.float32)
    p = O.OracleParams(n=n, R=R, L=L, r_max_cell=0.004)
    lab, _, _ = O.jfa_labels(pos, rad, p)
    cfg = FosConfig(DOMAIN_SIZE=L, CELL_SIZE=0.08, JFA_RES=R, JFA_RES_MIN=2, JFA_RES_MAX=R,
                    JFA_EARLY_EXIT_ENABLED=False, MAX_PARTICLES=n)
    ctx = Context(cfg, max_n=n, max_res=R)
    ctx.jfa_run(_dev(pos), _dev(rad), n)
    torch.cuda.synchronize()
    assert np.array_equal(ctx.labels().cpu().numpy().reshape(-1), lab)
    ids, cnt = O.accumulate_faces(O.majority_filter(lab, R), R, n)
    assert np.array_equal(ctx.face_ids[:n].cpu().numpy(), ids)
    assert np.array_equal(ctx.face_counts[:n].cpu().numpy(), cnt)
    prev = np.zeros((n, 32), np.float32)
    nl, used, fsc = O.finalize(rad, ids, cnt, prev, p)
    assert np.array_equal(ctx.fsc[:n].cpu().numpy(), fsc)
    assert np.array_equal(ctx.neighbor_list[:n].cpu().numpy(), nl)
    assert ctx.device_error() == 0


def test_early_exit_and_tie_rule_flags():
    foam = inputs.small()
    pos, rad = wrapped(foam.pos), foam.rad.copy()
    for early, tie in [(True, False), (False, True), (True, True)]:
        p = oracle_params(foam, early_exit=early, tie_lower=tie)
        lab, ch, done = O.jfa_labels(pos, rad, p)
        cfg, ctx = _ctx(foam, JFA_EARLY_EXIT_ENABLED=early, TIE_LOWER_INDEX=tie)
        ctx.jfa_run(_dev(pos), _dev(rad), foam.n)
        st = ctx.jfa_stats(foam.n, _dev(rad))
        V = float(p.R ** 3)
        fired = any(q >= p.min_passes - 1 and ch[q] / V < p.th_delta for q in range(done))
        # run_jfa sets early_exit when the exit test fires, even on the last pass
        assert st["num_passes"] == done and st["early_exit"] == (early and fired)
        assert np.array_equal(ctx.labels().cpu().numpy().reshape(-1), lab)


def test_coincident_seeds_tie_to_lowest_index():
    """Several seeds in one voxel at identical positions: argmin ties -> lowest i."""
    n = 6
    pos = np.zeros((n, 3), np.float32)
    pos[:3] = [0.1, 0.1, 0.1]
    pos[3:] = [-0.2, 0.3, 0.0]
    rad = np.full(n, 0.05, np.float32)
    R = 16
    p = O.OracleParams(n=n, R=R)
    lab = O.jfa_init(pos, rad, p)
    cfg = FosConfig(DOMAIN_SIZE=1.0, CELL_SIZE=0.1, JFA_RES=R, JFA_RES_MIN=2, JFA_RES_MAX=R,
                    JFA_EARLY_EXIT_ENABLED=False, MAX_PARTICLES=n)
    ctx = Context(cfg, max_n=n, max_res=R)
    ctx.jfa_init(_dev(pos), _dev(rad), n)
    torch.cuda.synchronize()
    g = ctx.labels()  # before passes the final buffer index is 0 -> init grid
    assert set(np.unique(lab)) == {-1, 0, 3}
    assert np.array_equal(g.cpu().numpy().reshape(-1), lab)
    ctx.jfa_passes(n)
    ctx.majority_filter()
    ctx.accumulate_faces(n)
    ctx.finalize(_dev(rad), n)
    torch.cuda.synchronize()
    full, _, _ = O.jfa_labels(pos, rad, p)
    assert np.array_equal(ctx.labels().cpu().numpy().reshape(-1), full)


@pytest.mark.parametrize("R", [32, 27, 20])
def test_stage_by_stage_with_loaded_labels(R):
    """FSC stages on a given owner grid (stripes + noise) match the oracle; R a
    multiple of 8 takes the face kernel's 2x2x8 warp tiles, 27 and 20 its
    linear voxel order."""
    rng = np.random.default_rng(2)
    n = 40
    lab = rng.integers(-1, n, (R, R, R)).astype(np.int32)
    lab[:, :, :16] = rng.integers(0, 5, (R, R, 16))
    lab = lab.reshape(-1)
    rad = rng.uniform(0.01, 0.03, n).astype(np.float32)
    p = O.OracleParams(n=n, R=R)
    cfg = FosConfig(DOMAIN_SIZE=1.0, CELL_SIZE=0.1, JFA_RES=R, JFA_RES_MIN=2, JFA_RES_MAX=R,
                    JFA_EARLY_EXIT_ENABLED=False, MAX_PARTICLES=n)
    ctx = Context(cfg, max_n=n, max_res=R)
    ctx.load_labels(_dev(lab))
    ctx.majority_filter()
    ctx.accumulate_faces(n)
    ctx.finalize(_dev(rad), n)
    ctx.update_ema(n)
    torch.cuda.synchronize()
    filt = O.majority_filter(lab, R)
    ids, cnt = O.accumulate_faces(filt, R, n)
    prev = np.zeros((n, 32), np.float32)
    nl, used, fsc = O.finalize(rad, ids, cnt, prev, p)
    ema = np.zeros(n, np.float32)
    O.fsc_ema(fsc, ema, p.ema_alpha)
    assert np.array_equal(ctx.label_filtered().cpu().numpy().reshape(-1), filt)
    assert np.array_equal(ctx.face_ids[:n].cpu().numpy(), ids)
    assert np.array_equal(ctx.face_counts[:n].cpu().numpy(), cnt)
    assert np.array_equal(ctx.fsc[:n].cpu().numpy(), fsc)
    assert np.array_equal(ctx.neighbor_list[:n].cpu().numpy(), nl)
    assert np.array_equal(ctx.neighbor_prev_scores[:n].cpu().numpy(), prev)
    assert np.array_equal(ctx.fsc_ema[:n].cpu().numpy(), ema)


def test_single_and_empty():
    R = 16
    cfg = FosConfig(DOMAIN_SIZE=1.0, CELL_SIZE=0.1, JFA_RES=R, JFA_RES_MIN=2, JFA_RES_MAX=R,
                    JFA_EARLY_EXIT_ENABLED=False, MAX_PARTICLES=4)
    ctx = Context(cfg, max_n=4, max_res=R)
    pos = _dev(np.array([[0.3, -0.2, 0.1]], np.float32))
    rad = _dev(np.array([0.05], np.float32))
    ctx.jfa_run(pos, rad, 1)
    torch.cuda.synchronize()
    assert bool((ctx.labels() == 0).all())
    assert int(ctx.fsc[0]) == 0
    ctx.jfa_run(pos, rad, 0)  # n = 0: all voxels unassigned, nothing else to do
    torch.cuda.synchronize()
    assert bool((ctx.labels() == -1).all())


def test_capacity_errors_are_loud():
    from fos import FosError
    R = 16
    cfg = FosConfig(DOMAIN_SIZE=1.0, CELL_SIZE=0.1, JFA_RES=R, JFA_RES_MIN=2, JFA_RES_MAX=R,
                    MAX_PARTICLES=4)
    ctx = Context(cfg, max_n=4, max_res=R)
    pos = torch.zeros((8, 3), dtype=torch.float32, device="cuda")
    rad = torch.full((8,), 0.01, dtype=torch.float32, device="cuda")
    with pytest.raises(FosError):
        ctx.jfa_run(pos, rad, 8)
    with pytest.raises(FosError):
        ctx.set_resolution(64)
    with pytest.raises(TypeError):
        ctx.jfa_run(pos.double(), rad, 2)


@pytest.mark.parametrize("shift", [0.0, 0.5, 1.75, 3.0e6])
def test_unwrapped_seed_positions(shift):
    """Seeds given outside [-L/2, L/2) (unwrapped or shifted by whole boxes) use
    the same jfa.wrapP arithmetic: labels match the oracle bit for bit.  The
    3e6 shift rounds positions to multiples of 0.25 (many exact distance ties)
    and takes the conversion-unit rounding path for huge coordinates."""
    rng = np.random.default_rng(21)
    n, R = 400, 32
    pos = (rng.random((n, 3), dtype=np.float32) - np.float32(0.5) + np.float32(shift))
    rad = rng.uniform(0.02, 0.05, n).astype(np.float32)
    p = O.OracleParams(n=n, R=R)
    lab, _, _ = O.jfa_labels(pos, rad, p)
    cfg = FosConfig(DOMAIN_SIZE=1.0, CELL_SIZE=0.1, JFA_RES=R, JFA_RES_MIN=2, JFA_RES_MAX=R,
                    JFA_EARLY_EXIT_ENABLED=False, MAX_PARTICLES=n)
    ctx = Context(cfg, max_n=n, max_res=R)
    ctx.jfa_run(_dev(pos), _dev(rad), n)
    torch.cuda.synchronize()
    assert np.array_equal(ctx.labels().cpu().numpy().reshape(-1), lab)


@pytest.mark.parametrize("R", [16, 32, 36, 48, 64, 96, 128, 256])
def test_pass_forms_agree(R):
    """The record pass with four voxels a thread along x (forced at every R),
    the one-voxel-a-thread pass and (R >= 32) the pass with TMA-staged rows
    give the same labels and per-pass change counts, with and without early
    exit; at R <= 48 the four-voxel pass is also checked against the oracle.
    R = 36, 48 and 96 take the multi-voxel pass for any R (two voxels a thread
    at the first step, four where R is a multiple of 4 steps, one voxel a
    thread at R = 36's step 4)."""
    rng = np.random.default_rng(R + 1)
    n = 40 + R * 4
    pos = wrapped(rng.random((n, 3), dtype=np.float32))
    rad = rng.uniform(0.5, 1.5, n).astype(np.float32) / R ** 0.5 * 0.2
    forms = [(2, False), (0, False)] + ([(0, True)] if R >= 32 else [])
    for early in (False, True):
        cfg = FosConfig(DOMAIN_SIZE=1.0, CELL_SIZE=0.1, JFA_RES=R, JFA_RES_MIN=2, JFA_RES_MAX=R,
                        JFA_EARLY_EXIT_ENABLED=early, MAX_PARTICLES=n)
        out = []
        for multi, staged in forms:
            ctx = Context(cfg, max_n=n, max_res=R)
            ctx.set_jfa_multi_voxel(multi)
            ctx.set_jfa_staging(staged)
            drad = _dev(rad)
            ctx.jfa_run(_dev(pos), drad, n)
            st = ctx.jfa_stats(n, drad)
            out.append((ctx.labels().cpu().numpy().reshape(-1), st["label_changes"],
                        st["num_passes"]))
            assert ctx.device_error() == 0
            ctx.close()
        for o in out[1:]:
            assert np.array_equal(out[0][0], o[0]) and out[0][1] == o[1] and out[0][2] == o[2]
        if R <= 48:
            p = O.OracleParams(n=n, R=R, early_exit=early, r_max_cell=0.05)
            lab, ch, done = O.jfa_labels(pos, rad, p)
            assert np.array_equal(out[0][0], lab) and done == out[0][2]
            assert out[0][1] == [int(c) for c in ch]


@pytest.mark.parametrize("R", [32, 64, 128, 256])
def test_staged_rows_equal_global_rows(R):
    """The pass with TMA-staged record rows (power-of-two R in 32..256) and the
    pass reading the rows from global memory give the same labels and the
    same per-pass change counts, with and without early exit; at R = 32 the
    staged pass is also checked against the oracle."""
    rng = np.random.default_rng(R)
    n = 40 + R * 4
    pos = wrapped(rng.random((n, 3), dtype=np.float32))
    rad = rng.uniform(0.5, 1.5, n).astype(np.float32) / R ** 0.5 * 0.2
    for early in (False, True):
        cfg = FosConfig(DOMAIN_SIZE=1.0, CELL_SIZE=0.1, JFA_RES=R, JFA_RES_MIN=2, JFA_RES_MAX=R,
                        JFA_EARLY_EXIT_ENABLED=early, MAX_PARTICLES=n)
        out = []
        for staged in (True, False):
            ctx = Context(cfg, max_n=n, max_res=R)
            ctx.set_jfa_staging(staged)
            dpos, drad = _dev(pos), _dev(rad)
            ctx.jfa_run(dpos, drad, n)
            st = ctx.jfa_stats(n, drad)
            out.append((ctx.labels().cpu().numpy().reshape(-1), st["label_changes"],
                        st["num_passes"], ctx.fsc[:n].cpu().numpy()))
            assert ctx.device_error() == 0
            ctx.close()
        assert np.array_equal(out[0][0], out[1][0])
        assert out[0][1] == out[1][1] and out[0][2] == out[1][2]
        assert np.array_equal(out[0][3], out[1][3])
        if R == 32:
            p = O.OracleParams(n=n, R=R, early_exit=early, r_max_cell=0.05)
            lab, ch, done = O.jfa_labels(pos, rad, p)
            assert np.array_equal(out[0][0], lab) and done == out[0][2]
