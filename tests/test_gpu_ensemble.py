"""GPU checks of batched ensembles (no reference counterpart; the checker is
the single-foam path, itself held bit-exact to the oracle).

Bar: after every frame, each foam of the ensemble equals the same foam run
alone through FoamSim bit for bit: positions, radii, radius targets, fsc,
fsc_ema, face_ids and neighbour lists (renumbered to the foam's own indices).
Launch shapes (any tuning) and graph replay do not change a bit.
"""
import numpy as np
import pytest
import torch

from fos import inputs
from fos.driver import FoamSim
from fos.ensemble import FIXED, REPORT_KEYS, Ensemble

pytestmark = pytest.mark.gpu

# warm start of 2 JFA frames then JFA every 3rd, controller gate open from
# frame 2, so a few frames cover JFA and plain frames, targets and the nudge
OVER = dict(JFA_WARM_FRAMES=2, JFA_CADENCE=3, WARMSTART_FRAMES=2)


def _foams():
    # 64^3 (pow2), 96^3 (non-pow2) and 128^3 grids, different bands and seeds
    return [inputs.ensemble_member(700, 11, 10), inputs.ensemble_member(3000, 12, 12),
            inputs.ensemble_member(9000, 13, 14)]


def _singles(foams):
    sims = [FoamSim.from_foam(f, **OVER) for f in foams]
    for s in sims:
        s.initialize()
    return sims


def _assert_same(ens, sims, where, rows=True):
    """rows=False before any JFA frame: face_ids then still hold the zeros of
    the reference's zero-initialised field, which are not particle indices."""
    for k, sim in enumerate(sims):
        got = ens.foam(k)
        want = {"pos": sim.pos, "rad": sim.rad, "rad_target": sim.rad_target, "fsc": sim.fsc,
                "fsc_ema": sim.fsc_ema}
        if rows:
            want.update(face_ids=sim.face_ids, neighbor_list=sim.neighbor_list)
        for key, w in want.items():
            g = got[key]
            assert torch.equal(g, w), f"{where}: foam {k} {key} differs " \
                f"({(g != w).sum().item()} entries)"


def test_resolutions_follow_the_rule():
    foams = _foams()
    assert [f.res for f in foams] == [64, 96, 128]


@pytest.mark.parametrize("use_graph", [True, False])
def test_ensemble_equals_single_foams(use_graph):
    foams = _foams()
    ens = Ensemble(foams, **OVER)
    ens.use_graph = use_graph
    sims = _singles(foams)
    ens.initialize()
    torch.cuda.synchronize()
    _assert_same(ens, sims, "after init", rows=False)
    for f in range(8):
        jfa = ens.step()
        for s in sims:
            assert s.step() == jfa
        torch.cuda.synchronize()
        _assert_same(ens, sims, f"frame {f}")
    for s in sims:
        s.ctx.close()
    ens.close()


def test_ensemble_with_crowded_cells_equals_single_foams():
    """A foam that starts with 300 of its 2,000 particles in a 0.02 cube
    (hash cells 0.04 wide): its cells overflow the 32-slot rows, so those
    rebuilds of the ensemble's frame take the CSR form, and every foam still
    equals the same foam run alone."""
    from fos.inputs import Foam
    rng = np.random.default_rng(9)
    n = 2000
    pos = rng.random((n, 3), dtype=np.float32)
    pos[:300] = (0.3 + 0.02 * rng.random((300, 3))).astype(np.float32)
    rad = rng.uniform(0.01, 0.02, n).astype(np.float32)
    crowd = Foam("crowd-2k-64", pos, rad, 64, 0.01, 0.02, 10, 14, 8, 20, 20, 5, 500, 9)
    foams = [inputs.ensemble_member(700, 11, 10), crowd]
    ens = Ensemble(foams, **OVER)
    sims = _singles(foams)
    ens.initialize()
    for f in range(4):
        jfa = ens.step()
        for s in sims:
            assert s.step() == jfa
        torch.cuda.synchronize()
        _assert_same(ens, sims, f"frame {f}")
    for s in sims:
        s.ctx.close()
    ens.close()


def test_ensemble_with_ou_jitter_equals_single_foams():
    """The OU jitter (dynamics.py:607-660, run.py:855-867) inside the
    ensemble's dynamics kernel: each foam's mean radius from its own exact
    radius sum, its own Philox key and local counter, so every foam still
    equals the same foam run alone with the jitter on."""
    foams = _foams()
    over = dict(OVER, JITTER_ENABLED=True)
    ens = Ensemble(foams, **over)
    sims = [FoamSim.from_foam(f, **over) for f in foams]
    for s in sims:
        s.initialize()
    ens.initialize()
    for f in range(6):
        jfa = ens.step()
        for s in sims:
            assert s.step() == jfa
        torch.cuda.synchronize()
        _assert_same(ens, sims, f"frame {f}")
    for s in sims:
        s.ctx.close()
    ens.close()


def test_tuning_does_not_change_results():
    foams = _foams()
    outs = []
    tunings = [FIXED, {"pass_block": 128, "voxel_block": 512, "coop_threads": 512,
                       "coop_blocks_per_sm": 2}]
    for t in tunings:
        ens = Ensemble(foams, **OVER)
        ens.tuning = t
        ens.initialize()
        ens.run(7)
        torch.cuda.synchronize()
        outs.append([ens.pos.clone(), ens.rad.clone(), ens.fsc.clone(), ens.neighbor_list.clone()])
        ens.close()
    for a, b in zip(*outs):
        assert torch.equal(a, b)


def test_autotune_reports_and_keeps_state(tmp_path):
    foams = _foams()
    ens = Ensemble(foams, **OVER)
    ref = Ensemble(foams, **OVER)
    for e in (ens, ref):
        e.initialize()
        e.run(4)
    cache = str(tmp_path / "tune.json")
    tuning, report = ens.autotune(reps=2, cache=cache)
    assert set(report) == set(REPORT_KEYS)
    assert all(v > 0 or v == -1 for v in report.values())
    assert report["coop=1024x1"] > 0
    assert tuning["pass_block"] in (128, 256, 512)
    # the tuner restores the dynamics state it timed on
    torch.cuda.synchronize()
    assert torch.equal(ens.pos, ref.pos) and torch.equal(ens.rad, ref.rad)
    for e in (ens, ref):
        e.run(3)
    torch.cuda.synchronize()
    assert torch.equal(ens.pos, ref.pos) and torch.equal(ens.fsc, ref.fsc)
    # a second ensemble of the same shape reuses the cached choice
    again = Ensemble(foams, **OVER)
    t2, r2 = again.autotune(cache=cache)
    assert t2 == tuning and r2 == report
    for e in (ens, ref, again):
        e.close()


def test_rejects_invalid_configurations():
    from fos import _lib
    with pytest.raises(_lib.FosError):
        Ensemble(_foams()[:1], MAX_EQ_NEI=20)
    ens = Ensemble(_foams()[:1], **OVER)
    with pytest.raises(_lib.FosError):
        ens.tuning = dict(FIXED, pass_block=96)
    ens.close()


@pytest.mark.parametrize("mode", ["anchored", "absolute"])
def test_ensemble_with_surrogate_equals_single_foams(mode):
    """The learned FSC surrogate between JFA frames inside the ensemble
    (fos_ensemble_frame_surrogate): pairs on each foam's own grid, the same
    model, mode and refresh schedule, so every foam equals the same foam run
    alone with the surrogate, through surrogate frames, plain frames (the
    policy's surrogate_every) and judged JFA frames."""
    import math

    from fos import surrogate as S
    sur = S.Surrogate(seed=3)

    def policy():
        return S.RefreshPolicy(every=3, warm_frames=2, surrogate_every=2, min_exact=0.0,
                               max_mean_abs_err=math.inf)
    foams = _foams()
    ens = Ensemble(foams, **OVER)
    ens.attach_surrogate(sur, policy(), mode)
    sims = [FoamSim.from_foam(f, surrogate=sur, policy=policy(), surrogate_mode=mode, **OVER)
            for f in foams]
    for s in sims:
        s.initialize()
    ens.initialize()
    for f in range(10):
        jfa = ens.step()
        for s in sims:
            assert s.step() == jfa
        torch.cuda.synchronize()
        _assert_same(ens, sims, f"frame {f}")
    st = ens.surrogate_stats()
    assert st["judged"] == sum(f.n for f in foams)
    assert st["pairs"] > 0 and ens.policy.judged
    for s in sims:
        s.ctx.close()
    ens.close()
