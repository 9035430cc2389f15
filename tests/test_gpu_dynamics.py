"""GPU parity of the dynamics kernels against the oracle.

Bar (FP32): positions, radii, volumes within 1e-5 relative (PBD, pressure,
controller); Brownian jitter and the max-overlap reduction are compared
exactly; the pressure kernel's powers (two products for r^3, a corrected
cbrtf for the 1/3 root) differ from libm powf by a few ulp, so it is held to
the 1e-5 relative tolerance, not bit equality.
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
RTOL = 1e-5


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def _grid(ctx, cfg, pos, n):
    G3 = cfg.grid_res() ** 3
    cc = torch.zeros(G3, dtype=torch.int32, device="cuda")
    cs = torch.zeros_like(cc)
    ci = torch.zeros(n, dtype=torch.int32, device="cuda")
    ctx.grid_build(pos, n, cc, cs, ci)
    return cc, cs, ci


def _pos_close(a, b):
    d = a - b
    d = d - np.round(d)  # periodic
    return np.max(np.abs(d)) <= RTOL * 0.5


@pytest.mark.parametrize("name", ["small", "headline"])
def test_pbd_and_max_overlap(name):
    foam = {"small": inputs.small, "headline": inputs.headline}[name]()
    p = oracle_params(foam)
    pos = wrapped(foam.pos)
    rad = foam.rad.copy()
    grid = O.grid_build(pos, p)
    omax, lmd = O.max_overlap(pos, rad, grid, p)
    out = O.pbd(pos, rad, grid, p)
    cfg = FosConfig.for_foam(foam)
    ctx = Context(cfg, max_n=foam.n, max_res=cfg.JFA_RES)
    dpos, drad = _dev(pos), _dev(rad)
    cc, cs, ci = _grid(ctx, cfg, dpos, foam.n)
    glmd = torch.zeros(foam.n, dtype=torch.float32, device="cuda")
    gmax = ctx.compute_max_overlap(dpos, drad, cs, cc, ci, glmd, foam.n)
    assert gmax == omax
    assert np.array_equal(glmd.cpu().numpy(), lmd)
    ctx.project_overlaps(dpos, drad, cs, cc, ci, foam.n)
    torch.cuda.synchronize()
    g = dpos.cpu().numpy()
    assert _pos_close(g, out)
    assert np.array_equal(g, out)  # same op order, IEEE sqrt/div: expected bitwise


@pytest.mark.parametrize("sweeps", [1, 10, 20])
def test_pressure_sweeps(sweeps):
    foam = inputs.headline()
    p = oracle_params(foam)
    pos = wrapped(foam.pos)
    rad = foam.rad.copy()
    lab, _, _ = O.jfa_labels(pos, rad, p)
    ids, cnt = O.accumulate_faces(O.majority_filter(lab, p.R), p.R, foam.n)
    prev = np.zeros((foam.n, 32), np.float32)
    nl, used, fsc = O.finalize(rad, ids, cnt, prev, p)
    r_o = rad.copy()
    for _ in range(sweeps):
        mx, ch, dr = O.pressure(r_o, ids, fsc, 37, p)
    cfg = FosConfig.for_foam(foam)
    ctx = Context(cfg, max_n=foam.n, max_res=cfg.JFA_RES)
    drad = _dev(rad)
    ddr = torch.zeros(foam.n, dtype=torch.float32, device="cuda")
    gmx, gch = ctx.equilibrate_pressure(foam.n, 37, drad, ddr, _dev(ids), _dev(fsc), p.k, p.P,
                                        p.pair_cap, p.max_nei, p.r_min, p.r_max, sweeps=sweeps)
    g = drad.cpu().numpy()
    assert np.max(np.abs(g - r_o) / r_o) <= RTOL
    assert abs(gmx - mx) <= RTOL * abs(mx) + 1e-12
    assert abs(gch - ch) <= max(2, ch // 1000)
    vol_g, vol_o = g.astype(np.float64) ** 3, r_o.astype(np.float64) ** 3
    assert np.max(np.abs(vol_g - vol_o) / vol_o) <= 3 * RTOL


def test_brownian_bit_exact():
    foam = inputs.headline()
    p = oracle_params(foam)
    pos = wrapped(foam.pos)
    o = pos.copy()
    O.brownian(o, p, 123)
    cfg = FosConfig.for_foam(foam)
    ctx = Context(cfg, max_n=foam.n, max_res=cfg.JFA_RES)
    d = _dev(pos)
    ctx.apply_brownian(d, foam.n, p.brownian, p.L, p.seed, 123)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), o)


def test_controller_kernels():
    foam = inputs.headline()
    p = oracle_params(foam)
    rng = np.random.default_rng(3)
    n = foam.n
    rad = foam.rad.copy()
    fsc = rng.integers(0, 25, n).astype(np.int32)
    ema = (fsc + rng.normal(0, 1.5, n)).astype(np.float32)
    ema[::7] = 0.0
    tgt = np.zeros(n, np.float32)
    O.set_targets(rad, tgt, fsc, ema, p)
    lmd = rng.uniform(0, 0.05, n).astype(np.float32)
    r2 = rad.copy()
    O.nudge(r2, tgt, lmd, 0.01, p)
    cfg = FosConfig.for_foam(foam)
    ctx = Context(cfg, max_n=n, max_res=cfg.JFA_RES)
    drad, dtgt = _dev(rad), torch.zeros(n, dtype=torch.float32, device="cuda")
    ctx.set_fsc_targets(drad, dtgt, _dev(fsc), _dev(ema), n, p.f_low, p.f_high, p.growth,
                        p.r_min, p.r_max)
    assert np.array_equal(dtgt.cpu().numpy(), tgt)
    alpha = np.float32(O.alpha_for_frames(p.adjust_frames))
    back = O.backpressure_from_overlap(0.01, p.contact_tol)
    ctx.nudge_radii(drad, dtgt, _dev(lmd), n, alpha, p.max_step, p.r_min, p.r_max, back,
                    p.bp_mode)
    torch.cuda.synchronize()
    assert np.array_equal(drad.cpu().numpy(), r2)
    g, s, i, md, mx = ctx.controller_stats(drad, dtgt, _dev(ema), n, p.f_low, p.f_high)
    assert g + s + i == n
    assert g == int(np.sum(ema < p.f_low)) and s == int(np.sum(ema > p.f_high))
    rmin, rmax = ctx.pressure_stats(n, drad)
    assert rmin == r2.min() and rmax == r2.max()
