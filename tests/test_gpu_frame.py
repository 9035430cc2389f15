"""Whole-frame parity: the GPU frame driver against the oracle's frame driver.

Frame 0 involves no power-dependent step (pressure is a no-op before the first
JFA), so it must be bit-exact end to end.  Later frames run the pressure
sweeps (their powers differ from libm powf by a few ulp): positions and radii are
held to 1e-5 relative after one frame, and longer runs are compared through
the FSC histogram and the radius distribution, since trajectories diverge.
"""
import numpy as np
import pytest
import torch

from fos import inputs
from fos.driver import FoamSim
from oracle import oracle as O

from helpers import oracle_params

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _pair(name, use_graph=True):
    foam = {"small": inputs.small, "headline": inputs.headline, "stress": inputs.stress}[name]()
    osim = O.OracleSim(oracle_params(foam), foam.pos, foam.rad)
    osim.initialize()
    gsim = FoamSim.from_foam(foam, use_graph=use_graph)
    gsim.initialize()
    return foam, osim, gsim


def _periodic_maxdiff(a, b):
    d = a - b
    d = d - np.round(d)
    return float(np.max(np.abs(d)))


@pytest.mark.parametrize("name,use_graph", [("small", False), ("small", True),
                                            ("stress", True)])
def test_initialisation_and_first_frame_bit_exact(name, use_graph):
    foam, osim, gsim = _pair(name, use_graph)
    torch.cuda.synchronize()
    assert np.array_equal(gsim.pos.cpu().numpy(), osim.pos)
    osim.step()
    gsim.step()
    torch.cuda.synchronize()
    assert np.array_equal(gsim.pos.cpu().numpy(), osim.pos)
    assert np.array_equal(gsim.rad.cpu().numpy(), osim.rad)
    assert np.array_equal(gsim.fsc.cpu().numpy(), osim.fsc)
    assert np.array_equal(gsim.neighbor_list.cpu().numpy(), osim.nl)
    assert np.array_equal(gsim.face_ids.cpu().numpy(), osim.face_ids)
    assert np.array_equal(gsim.fsc_ema.cpu().numpy(), osim.ema)
    f, settle = gsim.counters()
    assert f == 1 and settle == osim.settle


@pytest.mark.parametrize("name", ["small", "headline"])
def test_second_frame_within_tolerance(name):
    foam, osim, gsim = _pair(name)
    for _ in range(2):
        osim.step()
        gsim.step()
    torch.cuda.synchronize()
    r_g, r_o = gsim.rad.cpu().numpy(), osim.rad
    assert np.max(np.abs(r_g - r_o) / r_o) <= RTOL
    assert _periodic_maxdiff(gsim.pos.cpu().numpy(), osim.pos) <= RTOL
    vol_g, vol_o = r_g.astype(np.float64) ** 3, r_o.astype(np.float64) ** 3
    assert np.max(np.abs(vol_g - vol_o) / vol_o) <= 3 * RTOL
    agree = np.mean(gsim.fsc.cpu().numpy() == osim.fsc)
    assert agree >= 0.999


def test_long_run_distributions():
    """40 frames of the 1k foam (controller active after the 30-frame warm start)."""
    foam, osim, gsim = _pair("small")
    for _ in range(40):
        osim.step()
        gsim.step()
    torch.cuda.synchronize()
    fg, fo = gsim.fsc.cpu().numpy(), osim.fsc
    hg = np.bincount(fg, minlength=40)[:40] / len(fg)
    ho = np.bincount(fo, minlength=40)[:40] / len(fo)
    assert 0.5 * np.abs(hg - ho).sum() <= 0.05  # total-variation distance of FSC histograms
    rg, ro = np.sort(gsim.rad.cpu().numpy()), np.sort(osim.rad)
    allv = np.sort(np.concatenate([rg, ro]))
    ks = np.max(np.abs(np.searchsorted(rg, allv, "right") / len(rg)
                       - np.searchsorted(ro, allv, "right") / len(ro)))
    assert ks <= 0.05


@pytest.mark.parametrize("name", ["small", "headline", "stress"])
def test_cooperative_frame_matches_stage_kernels(name):
    """The persistent cooperative frame kernel and the one-kernel-per-stage path
    (used by the per-stage profiler) give bit-identical frames.  The 200k foam
    (175,616 cells) takes the chunked four-phase grid rebuild."""
    foam = {"small": inputs.small, "headline": inputs.headline, "stress": inputs.stress}[name]()
    a = FoamSim.from_foam(foam, use_graph=True)
    b = FoamSim.from_foam(foam, use_graph=False)
    a.initialize()
    b.initialize()
    for _ in range(6):
        a.step()
        b.step_profiled()
    torch.cuda.synchronize()
    assert np.array_equal(a.pos.cpu().numpy(), b.pos.cpu().numpy())
    assert np.array_equal(a.rad.cpu().numpy(), b.rad.cpu().numpy())
    assert np.array_equal(a.fsc.cpu().numpy(), b.fsc.cpu().numpy())
    assert np.array_equal(a.cell_indices.cpu().numpy(), b.cell_indices.cpu().numpy())
    assert np.array_equal(a.cell_start.cpu().numpy(), b.cell_start.cpu().numpy())
    assert np.array_equal(a.local_max_depth.cpu().numpy(), b.local_max_depth.cpu().numpy())
    assert a.counters() == b.counters()
    assert a.ctx.device_error() == 0


def test_cooperative_frame_with_crowded_cells():
    """Cells of more than 32 particles overflow the cooperative kernel's
    fixed-capacity rows, and those rebuilds take the CSR form; the frames still
    equal the one-kernel-per-stage path bit for bit.  300 particles start in a
    0.02 cube (hash cells 0.04 wide), so the first frames overflow."""
    from fos.inputs import Foam
    rng = np.random.default_rng(9)
    n = 2000
    pos = rng.random((n, 3), dtype=np.float32)
    pos[:300] = (0.3 + 0.02 * rng.random((300, 3))).astype(np.float32)
    rad = rng.uniform(0.01, 0.02, n).astype(np.float32)
    foam = Foam("crowd-2k-64", pos, rad, 64, 0.01, 0.02, 10, 16, 4, 10, 2, 2, 6, 5)
    a = FoamSim.from_foam(foam, use_graph=True)
    b = FoamSim.from_foam(foam, use_graph=False)
    a.initialize()
    b.initialize()
    for _ in range(4):
        a.step()
        b.step_profiled()
    torch.cuda.synchronize()
    for key in ("pos", "rad", "fsc", "cell_indices", "cell_start", "local_max_depth"):
        assert torch.equal(getattr(a, key), getattr(b, key)), key
    assert a.counters() == b.counters()
    assert a.ctx.device_error() == 0


@pytest.mark.parametrize("sweeps", [1, 7, 65])
def test_cooperative_pressure_sweep_counts(sweeps):
    """The cooperative kernel runs the pressure sweeps without grid barriers
    (tagged per-sweep words) for 1..64 sweeps and with a barrier per sweep
    beyond; both equal the one-kernel-per-stage path bit for bit."""
    import dataclasses
    foam = dataclasses.replace(inputs.small(), pressure_iters=sweeps)
    a = FoamSim.from_foam(foam, use_graph=True)
    b = FoamSim.from_foam(foam, use_graph=False)
    a.initialize()
    b.initialize()
    for _ in range(3):
        a.step()
        b.step_profiled()
    torch.cuda.synchronize()
    for key in ("pos", "rad", "fsc", "delta_r", "cell_indices"):
        assert torch.equal(getattr(a, key), getattr(b, key)), key
    assert a.counters() == b.counters()
    assert a.ctx.device_error() == 0


@pytest.mark.parametrize("r_max,G", [(0.2, 3), (0.13, 4), (0.11, 5)])
def test_cooperative_frame_on_coarse_grids(r_max, G):
    """Hash grids of 3 to 5 cells a side: the stencil wraps onto itself below 3
    distinct neighbours, and the stencil pruning of PBD / max overlap is off
    below 5 cells (on at 5); the cooperative frame still equals the stage
    kernels bit for bit."""
    from fos.inputs import Foam
    rng = np.random.default_rng(G)
    n = 150
    pos = rng.random((n, 3), dtype=np.float32)
    rad = rng.uniform(0.4 * r_max, r_max, n).astype(np.float32)
    foam = Foam(f"coarse-{G}", pos, rad, 32, 0.3 * r_max, r_max, 6, 14, 4, 10, 2, 2, 6, G)
    a = FoamSim.from_foam(foam, use_graph=True)
    b = FoamSim.from_foam(foam, use_graph=False)
    assert a.cfg.grid_res() == G
    a.initialize()
    b.initialize()
    for _ in range(4):
        a.step()
        b.step_profiled()
    torch.cuda.synchronize()
    for key in ("pos", "rad", "fsc", "cell_indices", "local_max_depth"):
        assert torch.equal(getattr(a, key), getattr(b, key)), key
    assert a.counters() == b.counters()
    assert a.ctx.device_error() == 0


def test_dynamics_trace_and_span():
    """fos_frame_trace: block 0's stamps after every phase, in order, inside the
    kernel's span (earliest block start .. latest block end); the frame counter
    does not move; cap < 3 is an argument error."""
    import ctypes as C
    from fos import _lib
    from fos._lib import call
    from fos.context import stream
    s = FoamSim.from_foam(inputs.small())
    s.initialize()
    s.run(3)
    before = s.counters()
    cap = 64
    buf = (C.c_longlong * cap)()
    cnt = C.c_int()
    call("fos_frame_trace", s.ctx.h, C.byref(s.state), C.byref(s.fp), buf, cap, C.byref(cnt),
         stream())
    t = [buf[i] for i in range(cnt.value)]
    assert 8 <= len(t) <= cap - 2
    assert all(b >= a for a, b in zip(t, t[1:]))
    start = (~buf[cap - 2]) & 0xFFFFFFFFFFFFFFFF
    end = buf[cap - 1]
    assert start <= t[0] and t[-1] <= end
    assert 0 < end - start < 50_000_000  # ns
    assert s.counters() == before
    with pytest.raises(_lib.FosError):
        call("fos_frame_trace", s.ctx.h, C.byref(s.state), C.byref(s.fp), buf, 2, C.byref(cnt),
             stream())
