"""Host-side logic that needs no GPU: configuration folding, workloads, schedule."""
import ctypes as C
import math

import numpy as np
import pytest

from fos import inputs
from fos.config import FosConfig
from oracle import oracle as O


def test_grid_res_matches_reference_formula():
    # GRID_RES = max(3, ceil(L / CELL_SIZE)) (config.py:317)
    for foam, expect in ((inputs.small(), 15), (inputs.headline(), 17), (inputs.stress(), 56)):
        cfg = FosConfig.for_foam(foam)
        assert cfg.grid_res() == expect
        assert cfg.grid_res() == O.OracleParams(n=foam.n, r_max_cell=foam.r_max).G
    assert FosConfig(DOMAIN_SIZE=1.0, CELL_SIZE=10.0).grid_res() == 3


@pytest.mark.parametrize("R,passes", [(64, 7), (128, 8), (192, 9), (256, 9), (320, 10)])
def test_pass_count(R, passes):
    # JFA_NUM_PASSES = ceil(log2 R) + 1 (jfa.py:223)
    assert FosConfig().jfa_num_passes(R) == passes


def test_cadence_schedule():
    cfg = FosConfig.for_foam(inputs.headline())
    frames = [f for f in range(40) if cfg.is_jfa_frame(f)]
    assert frames == list(range(20)) + [20, 25, 30, 35]
    small = FosConfig.for_foam(inputs.small())
    assert all(small.is_jfa_frame(f) for f in range(100))


def test_params_structs_carry_python_doubles():
    cfg = FosConfig.for_foam(inputs.headline())
    p = cfg.params()
    assert p.gap_fraction == 0.015 and p.t_add == 0.15 and p.domain_size == 1.0
    assert p.early_exit == 0 and p.grid_res == 17
    fp = cfg.frame_params()
    assert fp.pbd_iters == 8 and fp.pressure_iters == 20 and fp.f_low == 12 and fp.f_high == 16
    assert fp.bp_mode == 2 and fp.seed == 1
    # the folded f32 constant the library computes from the double
    assert np.float32(1.0 + p.gap_fraction) == np.float32(1.015)


def test_workload_shapes_and_laws():
    s, h, st = inputs.small(), inputs.headline(), inputs.stress()
    assert (s.n, s.res) == (1000, 64) and (h.n, h.res) == (10000, 128)
    assert (st.n, st.res) == (200000, 256)
    for f in (s, h, st):
        assert f.pos.dtype == np.float32 and f.rad.dtype == np.float32
        assert np.all(f.pos >= 0) and np.all(f.pos < 1)
    assert s.rad.min() >= 0.025 and s.rad.max() <= 0.035
    assert h.rad.min() >= 0.007 and h.rad.max() <= 0.03
    assert abs(np.median(h.rad) - 0.015) < 0.001
    small_mode = st.rad < 0.006
    assert abs(small_mode.mean() - 0.5) < 0.01
    assert np.all((st.rad >= 0.004) & (st.rad <= 0.009))
    # deterministic
    assert np.array_equal(inputs.headline().pos, h.pos)


def test_ensemble_workload():
    foams = inputs.ensemble()
    assert len(foams) == 64
    for f in foams:
        assert 2000 <= f.n <= 20000
        assert f.res in (64, 96, 128)
        assert f.res ** 3 / f.n >= 100 or f.res == 128
        assert 10 <= f.f_low <= 14 and f.f_high == f.f_low + 4


def test_alpha_and_backpressure():
    from fos.dynamics import alpha_for_frames, backpressure_from_overlap
    assert math.isclose(alpha_for_frames(15), 1 - 0.05 ** (1 / 15))
    assert backpressure_from_overlap(0.0, 0.035) == 1.0
    assert backpressure_from_overlap(0.1, 0.035) == 0.25
    assert backpressure_from_overlap(0.1, 0.0) == 1.0


def test_context_refuses_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from fos import FosError
    from fos.context import Context
    with pytest.raises(FosError):
        Context(FosConfig())
