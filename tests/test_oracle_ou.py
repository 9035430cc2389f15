"""The oracle's OU jitter (dynamics.py:600-690, run.py:855-867) against a
line-by-line numpy float32 transcription of apply_brownian + integrate_jitter.

ti.random() has no reproducible stream outside Taichi, so the draws come from
the project's Philox-4x32-10 (counter (i, frame, 'OUJT', 0), key = seed); the
transcription reads them through orc_philox, so the check pins the C
restatement's arithmetic and operation order, not the random stream.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

f32 = np.float32
OU_STREAM = 0x4F554A54


def _draws(n, frame, seed):
    out = np.empty(4, np.uint32)
    r = np.empty((n, 3), np.float32)
    for i in range(n):
        O.lib().orc_philox(i, frame, OU_STREAM, 0, seed & 0xFFFFFFFF, seed >> 32, O._ptr(out))
        r[i] = (out[:3] >> 8).astype(np.float32) * f32(2.0 ** -24) - f32(0.5)
    return r


def _ou_numpy(pos, v_jit, rad, mean_r, dt, rms, tau, max_drift, gap, L, seed, frame):
    """apply_brownian (dynamics.py:607-646) then integrate_jitter
    (dynamics.py:649-660), one particle at a time in float32; Python-level
    constants fold in double as Taichi folds them."""
    n = len(rad)
    r = _draws(n, frame, seed)
    dt = f32(dt)
    t = max(1e-6, tau)
    sigma = (f32(rms) * f32(mean_r)) * f32(math.sqrt(2.0 / t))
    kick = sigma * np.sqrt(dt)
    capk = f32(max_drift * gap)
    pos, v_jit = pos.copy(), v_jit.copy()
    for i in range(n):
        v = v_jit[i].copy()
        v = v + ((-v / f32(t)) * dt + kick * r[i])
        cap = capk * (rad[i] + rad[i])
        ln = np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * dt
        if ln > cap:
            v = v * ((cap / max(f32(1e-6), ln)) / dt)
        v_jit[i] = v
        p = pos[i] + v * dt
        pos[i] = p - f32(L) * np.floor(p * f32(1.0 / L) + f32(0.5))
    return pos, v_jit


def _case(n, seed, big=False):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-0.5, 0.5, (n, 3)).astype(np.float32)
    pos[: n // 10, 0] = f32(0.4999999)  # wrap across the +x face
    rad = rng.uniform(0.005, 0.03, n).astype(np.float32)
    v = rng.normal(0, 0.5 if big else 1e-3, (n, 3)).astype(np.float32)
    return pos, rad, v


def test_mean_radius_is_the_exact_mean():
    rng = np.random.default_rng(3)
    for n in (1, 7, 1000, 50000):
        rad = rng.uniform(0.002, 0.04, n).astype(np.float32)
        want = f32(math.fsum(rad.astype(np.float64).tolist()) / n)
        assert O.mean_radius(rad, n) == want
        assert O.mean_radius(rad[::-1].copy(), n) == want  # order-free
    assert O.mean_radius(np.zeros(1, np.float32), 0) == 0.0


@pytest.mark.parametrize("big", [False, True])
def test_ou_step_matches_transcription(big):
    n, seed = 300, 0x1234_0000_0042
    pos, rad, v = _case(n, 5, big)
    p = O.OracleParams(n=n, seed=seed, ou=True, jitter_rms=0.1 if not big else 40.0)
    for frame in (0, 17):
        want_pos, want_v = _ou_numpy(pos, v, rad, O.mean_radius(rad, n), p.dt, p.jitter_rms,
                                     p.jitter_tau, p.max_drift, p.gap, p.L, seed, frame)
        got_pos, got_v = pos.copy(), v.copy()
        O.ou_jitter(got_pos, got_v, rad, p, frame)
        assert np.array_equal(got_v, want_v)
        assert np.array_equal(got_pos, want_pos)
        pos, v = got_pos, got_v


def test_ou_cap_bounds_every_step_and_wraps():
    """The reference rescales v by (cap / L) / dt with L = |v| dt, so a capped
    velocity has |v| = cap / dt^2 and moves a particle cap / dt per step (the
    docstring's "<= cap" is not what the code does); the restatement keeps the
    code's behaviour."""
    n = 2000
    pos, rad, v = _case(n, 8, big=True)
    p = O.OracleParams(n=n, seed=4, ou=True, jitter_rms=100.0)
    O.ou_jitter(pos, v, rad, p, 2)
    step = np.sqrt((v.astype(np.float64) ** 2).sum(1)) * p.dt
    cap = f32(p.max_drift * p.gap) * (rad + rad) / p.dt
    assert np.all(step <= cap * (1 + 1e-5))
    assert np.mean(step >= cap * (1 - 1e-5)) > 0.99  # the cap binds at this rms
    assert np.all(pos >= -0.5) and np.all(pos < 0.5)


def test_ou_without_noise_decays_velocity():
    n = 100
    pos, rad, v = _case(n, 9)
    p = O.OracleParams(n=n, seed=4, ou=True, jitter_rms=0.0, max_drift=1e9)
    v0 = v.copy()
    O.ou_jitter(pos, v, rad, p, 0)
    want = v0 + (-v0 / f32(1.0)) * f32(p.dt)
    assert np.array_equal(v, want)


def test_ou_draws_are_uniform_and_centred():
    r = _draws(20000, 5, 77)
    assert np.all(r >= -0.5) and np.all(r < 0.5)
    assert abs(float(r.mean())) < 0.01
    assert abs(float(r.var()) - 1.0 / 12.0) < 0.003


def test_oracle_frame_with_and_without_ou():
    from fos import inputs
    from helpers import oracle_params
    foam = inputs.small()
    a = O.OracleSim(oracle_params(foam), foam.pos, foam.rad)
    b = O.OracleSim(oracle_params(foam, ou=True), foam.pos, foam.rad)
    for s in (a, b):
        s.initialize()
        s.step()
    assert np.all(a.v_jit == 0)
    assert np.any(b.v_jit != 0)
    assert not np.array_equal(a.pos, b.pos)
    # one OU step moves a particle by at most the per-step cap (cap / dt, see above)
    d = b.pos.astype(np.float64) - a.pos
    d -= np.round(d)
    cap = f32(b.p.max_drift * b.p.gap) * (b.rad + b.rad) / b.p.dt
    assert np.all(np.sqrt((d ** 2).sum(1)) <= cap * 1.01 + 1e-6)
