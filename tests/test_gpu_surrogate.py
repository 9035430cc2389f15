"""GPU checks of the FSC surrogate's kernels.

The surrogate has no counterpart in the reference.  Its checkers restate the
definitions in include/fos.h on the CPU (tests/surrogate_ref.py):
* pair sets, normalised distances, histograms and features: bit-exact against
  a float32 brute force over all pairs;
* tensor-core inference: against a torch BF16-weight reference, |dp| <= 2e-3
  per pair (FP32 accumulation order and BF16 rounding of the hidden layer);
* the fused segment inference of the frame path equals the flat-row
  inference bit for bit on the same pairs;
* training: gradient within 1e-4 relative (+1e-6 absolute) of torch FP32
  autograd; two Adam steps equal to torch.optim.Adam's to 1e-6 on all but
  near-zero-gradient entries;
* per-particle FSC = sum of the pair probabilities at both ends (to 2^-20 per
  pair, the fixed-point quantum);
* surrogate frames: the dynamics of a frame are those of the plain frame; the
  refresh cadence and drift-forced refreshes follow the policy; the graph
  replay equals the direct calls.
"""
import math

import numpy as np
import pytest
import torch

from fos import inputs
from fos import surrogate as S
from fos.config import FosConfig
from fos.context import Context
from fos.driver import FoamSim

import surrogate_ref as R

pytestmark = pytest.mark.gpu


def _grid(foam, cutoff):
    cfg = FosConfig.for_foam(foam)
    ctx = Context(cfg, max_n=foam.n, max_res=cfg.JFA_RES)
    ctx.set_resolution(cfg.JFA_RES)
    G3 = cfg.grid_res() ** 3
    z = lambda k: torch.zeros(k, dtype=torch.int32, device="cuda")
    cc, cs, ci = z(G3), z(G3), z(foam.n)
    pos = torch.as_tensor(np.ascontiguousarray(foam.pos, np.float32)).cuda()
    rad = torch.as_tensor(np.ascontiguousarray(foam.rad, np.float32)).cuda()
    ctx.grid_build(pos, foam.n, cc, cs, ci)  # wraps pos in place
    sur = S.Surrogate(cutoff=cutoff)
    return cfg, ctx, sur, pos, rad, cc, cs, ci


def _tiny_foam(seed=5, n=150):
    """Few, large particles: 10 hash cells per axis, so a 4.5 cutoff spans the axis."""
    rng = np.random.default_rng(seed)
    pos = rng.random((n, 3), dtype=np.float32)
    rad = rng.uniform(0.04, 0.05, n).astype(np.float32)
    return inputs.Foam("tiny", pos, rad, 64, 0.02, 0.05, 10, 16, 4, 10, 1 << 30, 1, 10, seed)


def _sorted(i, j, *cols):
    o = np.lexsort((j, i))
    return (i[o], j[o]) + tuple(c[o] for c in cols)


@pytest.mark.parametrize("case", ["small", "headline", "tiny-wide"])
def test_pairs_and_features_bit_exact(case):
    if case == "small":
        foam, cutoff = inputs.small(), 2.5
    elif case == "headline":
        foam, cutoff = inputs.headline(), 2.5
    else:
        foam, cutoff = _tiny_foam(), 4.5
    cfg, ctx, sur, pos, rad, cc, cs, ci = _grid(foam, cutoff)
    if case == "tiny-wide":
        G = cfg.grid_res()
        reach = int(np.floor(cutoff * (0.05 + foam.r_max) / (1.0 / G))) + 1
        assert 2 * reach + 1 >= G  # exercises the whole-axis branch
    ctx.jfa_run(pos, rad, foam.n)  # the memory features' lists and fsc
    S.build_pairs(ctx, sur, pos, rad, foam.n, foam.r_max, cs, cc, ci)
    d = S.export(ctx, rad, labels=False)
    torch.cuda.synchronize()
    assert d["overflow"] == 0
    n = foam.n
    ref = R.pairs_and_features(pos.cpu().numpy(), rad.cpu().numpy(), cutoff,
                               nl=ctx.neighbor_list[:n].cpu().numpy(),
                               used=ctx.neighbor_used_count[:n].cpu().numpy(),
                               fsc=ctx.fsc[:n].cpu().numpy())
    assert 0 < ref["X"][:, 14].sum() < len(ref["X"])
    gi, gj, gX = _sorted(d["i"].cpu().numpy(), d["j"].cpu().numpy(), d["X"].cpu().numpy())
    ri, rj, rX = _sorted(ref["i"], ref["j"], ref["X"])
    assert len(gi) == len(ri) and len(ri) > 0
    assert np.array_equal(gi, ri) and np.array_equal(gj, rj)
    assert np.array_equal(gX.view(np.uint32), rX.view(np.uint32))
    # segments are in owner order: i is non-decreasing in export order
    assert np.all(np.diff(d["i"].cpu().numpy()) >= 0)
    # ownership is balanced: low indices own about half of their pairs too
    deg = ref["hist"].sum(1)
    own = np.bincount(ref["i"], minlength=foam.n)
    assert own.sum() * 2 == deg.sum()
    low = slice(0, foam.n // 10)
    assert 0.4 < own[low].sum() / deg[low].sum() < 0.6
    ctx.close()


def test_pair_overflow_is_counted():
    foam = _tiny_foam(n=900)  # ~250 candidates, ~125 owned per particle: above the cap
    cfg, ctx, sur, pos, rad, cc, cs, ci = _grid(foam, 4.5)
    S.build_pairs(ctx, sur, pos, rad, foam.n, foam.r_max, cs, cc, ci)
    P, overflow = S.pair_count(ctx)
    ref = R.pairs_and_features(pos.cpu().numpy(), rad.cpu().numpy(), 4.5)
    per_i = np.bincount(ref["i"], minlength=foam.n)
    assert overflow == int((per_i > 96).sum()) > 0
    assert P == int(np.minimum(per_i, 96).sum())
    ctx.close()


def test_labels_follow_jfa_neighbor_lists():
    foam = inputs.small()
    cfg, ctx, sur, pos, rad, cc, cs, ci = _grid(foam, 2.5)
    ctx.jfa_run(pos, rad, foam.n)
    S.build_pairs(ctx, sur, pos, rad, foam.n, foam.r_max, cs, cc, ci)
    d = S.export(ctx, rad)
    nl = ctx.neighbor_list[: foam.n].cpu().numpy()
    i, j, y = d["i"].cpu().numpy(), d["j"].cpu().numpy(), d["y"].cpu().numpy()
    want = np.array([jj in set(nl[ii]) for ii, jj in zip(i, j)], np.float32)
    assert np.array_equal(y, want)
    assert 0 < y.sum() < len(y)
    ctx.close()


def _random_model(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    params = S.init_params(seed) * np.float32(scale)
    mu = rng.normal(0, 1, 16).astype(np.float32)
    sd = rng.uniform(0.5, 2.0, 16).astype(np.float32)
    return params, mu, sd


@pytest.mark.parametrize("P", [1, 15, 17, 1000, 40001])
def test_forward_matches_bf16_reference(P):
    params, mu, sd = _random_model(1, scale=3.0)
    sur = S.Surrogate()
    sur.set_weights(params, mu, sd)
    rng = np.random.default_rng(P)
    X = (rng.normal(0, 1.5, (P, 16)) * sd + mu).astype(np.float32)
    prob = sur.forward(torch.as_tensor(X).cuda()).cpu().numpy()
    ref = R.mlp_forward_bf16(X, params, mu, sd).numpy()
    err = np.abs(prob - ref)
    assert err.max() <= 2e-3, err.max()
    assert err.mean() <= 2e-4


@pytest.mark.parametrize("B", [64, 1000, 70000])
def test_gradient_matches_torch_fp32(B):
    params, mu, sd = _random_model(2)
    sur = S.Surrogate()
    sur.set_weights(params, mu, sd)
    rng = np.random.default_rng(B)
    Pn = B + 37
    X = (rng.normal(0, 1, (Pn, 16)) * sd + mu).astype(np.float32)
    y = (rng.random(Pn) < 0.4).astype(np.float32)
    rows = rng.permutation(Pn)[:B].astype(np.int32)
    g, loss = sur.gradient(torch.as_tensor(X).cuda(), torch.as_tensor(y).cuda(),
                           torch.as_tensor(rows).cuda())
    lt, pt = R.mlp_loss(X[rows], y[rows], params, mu, sd)
    lt.backward()
    gr = pt.grad.numpy()
    g = g.cpu().numpy()
    lv = float(lt.detach())
    assert abs(float(loss.item()) - lv) <= 1e-5 * max(1.0, abs(lv))
    assert np.allclose(g, gr, rtol=1e-4, atol=1e-6), np.abs(g - gr).max()


def test_adam_step_matches_torch():
    params, mu, sd = _random_model(3)
    sur = S.Surrogate()
    sur.set_weights(params, mu, sd)
    rng = np.random.default_rng(7)
    X = (rng.normal(0, 1, (5000, 16)) * sd + mu).astype(np.float32)
    y = (rng.random(5000) < 0.5).astype(np.float32)
    rows = np.arange(5000, dtype=np.int32)
    Xd, yd, rd = (torch.as_tensor(a).cuda() for a in (X, y, rows))
    lr = 1e-3
    for _ in range(2):
        sur.train_step(Xd, yd, rd, lr)
    got, _, _ = sur.get_weights()
    p = torch.tensor(params, requires_grad=True)
    opt = torch.optim.Adam([p], lr=lr, betas=(0.9, 0.999), eps=1e-8)
    for _ in range(2):
        opt.zero_grad()
        lt, pt = R.mlp_loss(X, y, p.detach().numpy(), mu, sd)
        lt.backward()
        p.grad = pt.grad
        opt.step()
    want = p.detach().numpy()
    close = np.abs(got - want) <= 1e-6
    assert close.mean() >= 0.995, close.mean()
    assert np.abs(got - want).max() <= 4 * lr


def test_training_learns_a_separable_rule():
    rng = np.random.default_rng(11)
    P = 200000
    X = rng.normal(0, 1, (P, 16)).astype(np.float32)
    y = ((X[:, 0] + 0.5 * X[:, 3] - X[:, 7] * X[:, 8]) > 0.2).astype(np.float32)
    Xd, yd = torch.as_tensor(X).cuda(), torch.as_tensor(y).cuda()
    sur = S.Surrogate()
    sur.standardize_from(Xd)
    losses = sur.fit(Xd, yd, epochs=15, batch=65536, lr=3e-3)
    assert losses[-1] < 0.5 * losses[0]
    acc = ((sur.forward(Xd) > 0.5).float() == yd).float().mean().item()
    assert acc > 0.93, acc


def test_predict_sums_pair_probabilities():
    foam = inputs.headline()
    cfg, ctx, sur, pos, rad, cc, cs, ci = _grid(foam, 2.5)
    params, _, _ = _random_model(4)
    sur.set_weights(params, np.zeros(16, np.float32) + 5.0, np.ones(16, np.float32) * 10.0)
    S.build_pairs(ctx, sur, pos, rad, foam.n, foam.r_max, cs, cc, ci)
    from fos._lib import call
    call("fos_surrogate_set_inference", ctx.h, 0)  # mma.sync: the same tiles as forward()
    out = S.predict(ctx, sur, rad, foam.n, with_pairs=True)
    d = S.export(ctx, rad, labels=False)
    P, _ = S.pair_count(ctx)
    prob = out["prob"][:P].cpu().numpy().astype(np.float64)
    i, j = d["i"].cpu().numpy(), d["j"].cpu().numpy()
    want = np.bincount(i, prob, foam.n) + np.bincount(j, prob, foam.n)
    got = out["fsc_float"].cpu().numpy()
    deg = np.bincount(i, minlength=foam.n) + np.bincount(j, minlength=foam.n)
    assert np.all(np.abs(got - want) <= deg * 2.0 ** -20 + 1e-5)
    assert np.array_equal(out["fsc"].cpu().numpy(), np.rint(got).astype(np.int32))
    # the flat-row tensor-core path on the exported rows gives the same bits
    prob2 = sur.forward(d["X"]).cpu().numpy()
    assert np.array_equal(prob2, prob.astype(np.float32))
    ctx.close()


def _sim(surrogate=None, policy=None, foam=None, **kw):
    foam = foam or inputs.small()
    return FoamSim.from_foam(foam, surrogate=surrogate, policy=policy, JFA_WARM_FRAMES=3,
                             JFA_CADENCE=5, **kw)


def test_surrogate_frame_keeps_plain_dynamics():
    """Within a frame the surrogate only changes rad_target / fsc_ema: the
    positions and radii after the frame equal the plain frame's."""
    sur = S.Surrogate()
    a = _sim()
    b = _sim(surrogate=sur, policy=S.RefreshPolicy(every=5, warm_frames=3))
    for sim in (a, b):
        sim.initialize()
    for f in range(4):
        a.step()
        b.step()
        torch.cuda.synchronize()
        assert torch.equal(a.pos, b.pos) and torch.equal(a.rad, b.rad), f
    assert not b.policy.judged  # frame 3 was a surrogate (non-JFA) frame
    a.ctx.close()
    b.ctx.close()


def test_refresh_cadence_judging_and_forced_refresh():
    foam = inputs.small()
    X = S.collect([foam], S.Surrogate(), export_frames=(2,))
    sur = S.Surrogate()
    sur.standardize_from(X["X"])
    sur.fit(X["X"], X["y"], epochs=5, batch=8192)
    # drift guard off: warm frames 0-2, then every 3rd frame
    calm = S.RefreshPolicy(every=3, warm_frames=3, min_exact=0.0, max_mean_abs_err=math.inf)
    sim = _sim(surrogate=sur, policy=calm, foam=foam)
    sim.initialize()
    jfa_frames = [f for f in range(12) if sim.step()]
    assert jfa_frames == [0, 1, 2, 5, 8, 11], jfa_frames
    assert calm.forced_total == 0 and len(calm.judged) == 3
    s = calm.judged[-1]
    assert s["judged"] == foam.n
    assert 0 <= s["exact"] <= s["within1"] <= foam.n
    assert s["stale_exact"] <= s["stale_within1"] <= foam.n
    sim.ctx.close()
    # an unreachable agreement threshold: the first judged frame (5) drifts and
    # every later frame is a forced refresh, each judged again
    pol = S.RefreshPolicy(every=3, warm_frames=3, min_exact=1.01, force_frames=2)
    sim = _sim(surrogate=sur, policy=pol, foam=foam)
    sim.initialize()
    jfa_frames = [f for f in range(12) if sim.step()]
    assert jfa_frames == [0, 1, 2, 5, 6, 7, 8, 9, 10, 11], jfa_frames
    assert pol.forced_total == len(pol.judged) == 7
    sim.ctx.close()


@pytest.mark.parametrize("mode", ["anchored", "absolute"])
def test_surrogate_graph_equals_direct(mode):
    sur = S.Surrogate(seed=3)
    outs = []
    for use_graph in (True, False):
        sim = FoamSim.from_foam(inputs.small(), use_graph=use_graph, surrogate=sur,
                                surrogate_mode=mode,
                                policy=S.RefreshPolicy(every=4, warm_frames=2, surrogate_every=2),
                                JFA_WARM_FRAMES=2, JFA_CADENCE=4)
        sim.initialize()
        for _ in range(11):
            sim.step()
        torch.cuda.synchronize()
        outs.append((sim.pos.clone(), sim.rad.clone(), sim.rad_target.clone(),
                     sim.fsc_ema.clone()))
        sim.ctx.close()
    for x, y in zip(*outs):
        assert torch.equal(x, y)


def test_tcgen05_inference_matches_mma_sync_and_reference():
    """The tcgen05 / TMEM inference (128-pair tiles, tcgen05.mma into tensor
    memory, tcgen05.ld back) against the mma.sync kernel on the same pairs and
    against the torch BF16 reference on the exported rows.  The two kernels
    sum in different FP32 orders, and a hidden unit can land on the other
    side of a BF16 rounding boundary, so they agree within the reference's
    tolerance, not bit for bit."""
    from fos._lib import call
    foam = inputs.headline()
    cfg, ctx, sur, pos, rad, cc, cs, ci = _grid(foam, 2.5)
    n = foam.n
    ctx.jfa_run(pos, rad, n)
    params, mu, sd = _random_model(4, scale=3.0)
    sur.set_weights(params, mu, sd)
    S.build_pairs(ctx, sur, pos, rad, n, foam.r_max, cs, cc, ci)
    call("fos_surrogate_set_inference", ctx.h, 0)
    seg = S.predict(ctx, sur, rad, n, with_pairs=True)
    call("fos_surrogate_set_inference", ctx.h, 1)
    tc = S.predict(ctx, sur, rad, n, with_pairs=True)
    torch.cuda.synchronize()
    assert ctx.device_error() == 0
    P, _ = S.pair_count(ctx)
    assert P > 100_000
    p_seg = seg["prob"][:P].cpu().numpy()
    p_tc = tc["prob"][:P].cpu().numpy()
    d = np.abs(p_tc - p_seg)
    assert d.max() <= 4e-3 and d.mean() <= 2e-5, (d.max(), d.mean())
    X = S.export(ctx, rad, labels=False)["X"].cpu().numpy()
    ref = R.mlp_forward_bf16(X, params, mu, sd).numpy()
    # the memory features (fsc sums) standardise to large values here, where a
    # BF16 rounding of an input or hidden unit moves a probability by up to
    # ~1e-2; the tcgen05 kernel stays as close to the reference as mma.sync
    err, err_seg = np.abs(p_tc - ref), np.abs(p_seg - ref)
    assert err.max() <= max(2e-3, 1.5 * err_seg.max()), (err.max(), err_seg.max())
    assert err.mean() <= 2e-4, err.mean()
    f = np.abs(tc["fsc_float"].cpu().numpy() - seg["fsc_float"].cpu().numpy())
    assert f.max() <= 0.02
    ctx.close()


def test_tcgen05_frames_run_clean():
    """Surrogate frames with the tcgen05 inference: graph capture, the TMEM
    allocation of every CTA freed (later frames allocate again), no device
    error."""
    from fos._lib import call
    sur = S.Surrogate(seed=3)
    sim = FoamSim.from_foam(inputs.small(), surrogate=sur, surrogate_mode="absolute",
                            policy=S.RefreshPolicy(every=4, warm_frames=2, min_exact=0.0,
                                                   max_mean_abs_err=math.inf),
                            JFA_WARM_FRAMES=2, JFA_CADENCE=4)
    call("fos_surrogate_set_inference", sim.ctx.h, 1)
    sim.initialize()
    for _ in range(12):
        sim.step()
    torch.cuda.synchronize()
    assert sim.ctx.device_error() == 0
    assert torch.isfinite(sim.fsc_ema).all()
    sim.ctx.close()
