"""Host logic of the FSC surrogate (no GPU): the refresh policy, the parameter
layout shared with include/fos.h, and the CPU references the GPU tests use."""
import math
import os
import re

import numpy as np
import pytest
import torch

from fos import _lib
from fos import surrogate as S

import surrogate_ref as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_define(name):
    src = open(os.path.join(ROOT, "include", "fos.h")).read()
    m = re.search(rf"#define {name} (.+?)(?:/\*|$)", src, flags=re.M)
    return eval(m.group(1))


def test_constants_match_header():
    assert _header_define("FOS_SUR_FEATURES") == _lib.SUR_FEATURES == 16
    assert _header_define("FOS_SUR_HIDDEN") == _lib.SUR_HIDDEN == 64
    assert _header_define("FOS_SUR_BINS") == _lib.SUR_BINS == 11
    assert _header_define("FOS_SUR_PAIR_CAP") == _lib.SUR_PAIR_CAP
    assert _header_define("FOS_SUR_NPARAM") == _lib.SUR_NPARAM == 5313
    assert _header_define("FOS_SUR_ABSOLUTE") == _lib.SUR_ABSOLUTE
    assert _header_define("FOS_SUR_ANCHORED") == _lib.SUR_ANCHORED
    assert 3 + _lib.SUR_BINS + 2 == _lib.SUR_FEATURES  # geometry, bins, memory


def test_param_layout_round_trip():
    p = S.init_params(0)
    assert p.shape == (S.NPARAM,) and p.dtype == np.float32
    u = S.unpack(p)
    assert u["W1"].shape == (64, 16) and u["W2"].shape == (64, 64) and u["w3"].shape == (64,)
    flat = np.concatenate([u["W1"].ravel(), u["b1"], u["W2"].ravel(), u["b2"], u["w3"], u["b3"]])
    assert np.array_equal(flat, p)
    assert np.abs(u["W1"]).max() <= 1 / math.sqrt(16) and np.abs(u["W2"]).max() <= 1 / 8


def test_refresh_policy_cadence_and_drift():
    pol = S.RefreshPolicy(every=4, warm_frames=2, min_exact=0.5, force_frames=2)
    seq = []
    for f in range(14):
        j = pol.is_jfa(f)
        seq.append(j)
        pol.ran(f, j)
        if j and f >= pol.warm_frames:
            # frame 5 drifts once, everything else agrees
            pol.observe({"exact_frac": 0.1 if f == 5 else 0.9, "mean_abs_err": 0.0})
    jfa = [f for f, j in enumerate(seq) if j]
    # warm 0,1; every 4th after the last JFA: 5; drift forces 6, 7; then 11
    assert jfa == [0, 1, 5, 6, 7, 11], jfa
    assert pol.forced_total == 1 and len(pol.judged) == 4


def test_refresh_policy_abs_error_threshold():
    pol = S.RefreshPolicy(every=10, warm_frames=0, max_mean_abs_err=1.0, force_frames=1)
    assert pol.is_jfa(0)
    pol.ran(0, True)
    assert pol.observe({"exact_frac": 1.0, "mean_abs_err": 1.5}) is True
    assert pol.is_jfa(1)
    pol.ran(1, True)
    assert pol.observe({"exact_frac": 1.0, "mean_abs_err": 0.5}) is False
    assert not pol.is_jfa(2) and pol.is_jfa(11)


def test_refresh_policy_defaults_are_the_target():
    """By default the guard holds the surrogate to the target: fewer than 99 %
    of cells agreeing, or a mean error above 0.05 faces, forces a refresh."""
    pol = S.RefreshPolicy()
    assert pol.min_exact == 0.99 and pol.max_mean_abs_err == 0.05
    assert pol.observe({"exact_frac": 0.985, "mean_abs_err": 0.0}) is True
    assert S.RefreshPolicy().observe({"exact_frac": 0.995, "mean_abs_err": 0.06}) is True
    assert S.RefreshPolicy().observe({"exact_frac": 0.995, "mean_abs_err": 0.01}) is False


def test_refresh_policy_surrogate_every():
    pol = S.RefreshPolicy(every=10, warm_frames=0, surrogate_every=3)
    pol.ran(0, True)
    assert [f for f in range(1, 10) if pol.is_surrogate(f)] == [3, 6, 9]
    assert S.RefreshPolicy().surrogate_every == 1


def test_pair_reference_small_case_by_hand():
    # two particles across the periodic boundary, one far away
    pos = np.array([[0.49, 0.0, 0.0], [-0.49, 0.0, 0.0], [0.0, 0.3, 0.0]], np.float32)
    rad = np.array([0.01, 0.01, 0.01], np.float32)
    ref = R.pairs_and_features(pos, rad, 2.5)
    assert list(ref["i"]) == [0] and list(ref["j"]) == [1]   # 0 + 1 odd: 0 owns
    assert abs(ref["nd"][0] - 1.0) < 1e-5          # |d| = 0.02 through the boundary
    assert ref["X"][0, 1] == 1.0 and ref["X"][0, 2] == 0.0
    # each histogram holds only the other particle, removed from the pair's features
    assert ref["hist"][0].sum() == 1 and ref["X"][0, 3:].sum() == 0
    assert R.owns(2, 4) is False and R.owns(4, 2) is True  # even sum: larger index owns


def test_torch_references_agree_in_fp32_limit():
    params = S.init_params(1)
    mu = np.zeros(16, np.float32)
    sd = np.ones(16, np.float32)
    X = np.random.default_rng(0).normal(0, 1, (64, 16)).astype(np.float32)
    y = np.zeros(64, np.float32)
    p_bf16 = R.mlp_forward_bf16(X, params, mu, sd).numpy()
    loss, _ = R.mlp_loss(X, y, params, mu, sd)
    # with y = 0, BCE = mean(-log(1 - p)); BF16 rounding moves p by < 1e-2
    assert abs(np.mean(-np.log1p(-p_bf16)) - float(loss.detach())) < 2e-2


def test_set_mode_rejects_unknown():
    with pytest.raises(ValueError):
        S.set_mode(None, "bogus")


def test_surrogate_requires_device():
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    with pytest.raises(_lib.FosError):
        S.Surrogate()
