"""OU jitter on the GPU (dynamics.py:600-690, run.py:855-867) against the oracle.

The standalone kernels (init_jitter_velocities, compute_mean_radius,
apply_brownian, integrate_jitter) and the frame's step 6B are bit-exact: the
mean radius is an exact fixed-point sum and the update uses only correctly
rounded float32 operations.  Whole frames with the jitter on are bit-exact on
frame 0 (no powf), and the cooperative frame kernel, which runs the jitter
inside the last PBD sweep, equals the one-kernel-per-stage path bit for bit.
"""
import numpy as np
import pytest
import torch

from fos import dynamics, inputs, runtime
from fos.config import FosConfig
from fos.driver import FoamSim
from oracle import oracle as O

from helpers import oracle_params

pytestmark = pytest.mark.gpu
f32 = np.float32


def _case(n, seed, big=False):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-0.5, 0.5, (n, 3)).astype(np.float32)
    pos[: n // 10, 0] = f32(0.4999999)
    rad = rng.uniform(0.005, 0.03, n).astype(np.float32)
    v = rng.normal(0, 0.5 if big else 1e-3, (n, 3)).astype(np.float32)
    return pos, rad, v


@pytest.mark.parametrize("big", [False, True])
def test_standalone_kernels_match_oracle(big):
    n, seed = 20000, 0x55AA_0000_0003
    rms = 40.0 if big else 0.1
    cfg = FosConfig(DOMAIN_SIZE=1.0, GRID_RES=16, JFA_RES=64, SEED=seed, JITTER_RMS=rms,
                    MAX_PARTICLES=n)
    runtime.configure(cfg)
    runtime.init(max_particles=n, max_res=64)
    pos, rad, v = _case(n, 11, big)
    p = O.OracleParams(n=n, seed=seed, ou=True, jitter_rms=rms)
    g_pos = torch.as_tensor(pos).cuda()
    g_rad = torch.as_tensor(rad).cuda()
    g_v = torch.as_tensor(v).cuda()
    mean = torch.zeros(1, dtype=torch.float32, device="cuda")
    dynamics.compute_mean_radius(g_rad, n, mean)
    torch.cuda.synchronize()
    assert mean.item() == O.mean_radius(rad, n)
    for call in range(3):
        dynamics.apply_brownian(g_v, g_rad, mean, n, cfg.DT)
        dynamics.integrate_jitter(g_pos, g_v, n, cfg.DT)
        O.ou_jitter(pos, v, rad, p, dynamics._jitter_calls - 1)
        torch.cuda.synchronize()
        assert np.array_equal(g_v.cpu().numpy(), v), f"v_jit differs at call {call}"
        assert np.array_equal(g_pos.cpu().numpy(), pos), f"pos differs at call {call}"
    dynamics.init_jitter_velocities(g_v, n)
    torch.cuda.synchronize()
    assert torch.count_nonzero(g_v).item() == 0


def _pair(name, use_graph=True, **over):
    foam = {"small": inputs.small, "headline": inputs.headline}[name]()
    osim = O.OracleSim(oracle_params(foam, ou=True, **over), foam.pos, foam.rad)
    osim.initialize()
    cfg_over = {"JITTER_ENABLED": True}
    if "jitter_rms" in over:
        cfg_over["JITTER_RMS"] = over["jitter_rms"]
    gsim = FoamSim.from_foam(foam, use_graph=use_graph, **cfg_over)
    gsim.initialize()
    return osim, gsim


@pytest.mark.parametrize("name,use_graph", [("small", False), ("small", True),
                                            ("headline", True)])
def test_first_frame_bit_exact_with_ou(name, use_graph):
    # a large rms makes the drift visible at frame 0 (v_jit starts at zero)
    osim, gsim = _pair(name, use_graph, jitter_rms=50.0)
    osim.step()
    gsim.step()
    torch.cuda.synchronize()
    assert np.any(osim.v_jit != 0)
    assert np.array_equal(gsim.v_jit.cpu().numpy(), osim.v_jit)
    assert np.array_equal(gsim.pos.cpu().numpy(), osim.pos)
    assert np.array_equal(gsim.cell_indices.cpu().numpy(), osim.grid[2])
    assert np.array_equal(gsim.fsc.cpu().numpy(), osim.fsc)
    assert np.array_equal(gsim.neighbor_list.cpu().numpy(), osim.nl)


def test_profiled_stage_reports_ou():
    _, gsim = _pair("small")
    ms = gsim.step_profiled()
    assert ms["ou_jitter"] > 0.0


@pytest.mark.parametrize("name", ["small", "headline"])
def test_cooperative_frame_matches_stage_kernels_with_ou(name):
    foam = {"small": inputs.small, "headline": inputs.headline}[name]()
    a = FoamSim.from_foam(foam, use_graph=True, JITTER_ENABLED=True, JITTER_RMS=5.0)
    b = FoamSim.from_foam(foam, use_graph=False, JITTER_ENABLED=True, JITTER_RMS=5.0)
    a.initialize()
    b.initialize()
    for _ in range(6):
        a.step()
        b.step_profiled()
    torch.cuda.synchronize()
    for key in ("pos", "rad", "v_jit", "fsc", "cell_indices", "cell_start"):
        assert torch.equal(getattr(a, key), getattr(b, key)), key
    assert a.counters() == b.counters()
    assert a.ctx.device_error() == 0


def test_ou_off_leaves_v_jit_untouched():
    foam = inputs.small()
    a = FoamSim.from_foam(foam)
    a.initialize()
    a.run(3)
    torch.cuda.synchronize()
    assert torch.count_nonzero(a.v_jit).item() == 0


def test_ensemble_ou_needs_a_pbd_sweep():
    """Ensembles run the OU jitter inside the last PBD sweep (as the
    single-foam frame does), so a configuration without PBD sweeps is
    rejected; with sweeps it is accepted (test_gpu_ensemble covers its
    results)."""
    from fos import _lib
    from fos.ensemble import Ensemble
    with pytest.raises(_lib.FosError):
        Ensemble([inputs.ensemble_member(700, 11, 10)], JITTER_ENABLED=True, PBD_ITERS=0)
    Ensemble([inputs.ensemble_member(700, 11, 10)], JITTER_ENABLED=True).close()
