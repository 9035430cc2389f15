"""The bounded device waits give up.

A cooperative kernel whose blocks wait on one another at grid barriers must
end on its own when one block never arrives: the waiting blocks record
FOS_E_TIMEOUT in the device error word and return, nothing faults and nothing
hangs, and once the error word is cleared the same context computes frames
bit-identical to a fresh context's.  fos_test_barrier_plan makes one block
leave at a chosen barrier and shortens the wait bound from ~1 s to ~1 ms, so
each failure takes milliseconds.  The reference has no counterpart (its only
watchdog, JFA_WATCHDOG_INTERVAL in config.py:174, is unused).
"""
import time

import numpy as np
import pytest
import torch

from fos import inputs
from fos.config import FosConfig
from fos.context import Context
from fos.driver import FoamSim

pytestmark = pytest.mark.gpu

FOS_E_TIMEOUT = 4


def _frames(sim, k):
    for _ in range(k):
        sim.step()
    torch.cuda.synchronize()


def _same_state(a, b):
    return (torch.equal(a.pos, b.pos) and torch.equal(a.rad, b.rad)
            and torch.equal(a.fsc, b.fsc))


def test_dynamics_kernel_wait_gives_up_and_context_recovers():
    foam = inputs.small()
    cfg = FosConfig.for_foam(foam)
    ref = FoamSim(cfg, foam.pos, foam.rad, use_graph=False)
    ref.initialize()
    _frames(ref, 3)
    sim = FoamSim(cfg, foam.pos, foam.rad, use_graph=False)
    sim.initialize()
    ctx = sim.ctx
    # the last block leaves the frame's dynamics kernel at its 5th grid barrier
    ctx.test_barrier_plan(5)
    t0 = time.perf_counter()
    _frames(sim, 1)
    dt = time.perf_counter() - t0
    assert ctx.device_error() == FOS_E_TIMEOUT
    assert dt < 0.5  # the ~1 ms bound, far below the 1 s one
    ctx.test_barrier_plan(0)
    ctx.clear_device_error()
    # the same context, fresh state: the frames equal a clean context's
    again = FoamSim(cfg, foam.pos, foam.rad, use_graph=False, ctx=ctx)
    again.initialize()
    _frames(again, 3)
    assert ctx.device_error() == 0
    assert _same_state(again, ref)
    ref.ctx.close()
    ctx.close()


def test_finalize_wait_gives_up_and_context_recovers():
    foam = inputs.headline()  # the finalize fixed point takes 2-3 sweeps here
    cfg = FosConfig.for_foam(foam)
    n = foam.n
    ctx = Context(cfg, max_n=n, max_res=cfg.JFA_RES)
    f = np.float32
    p = foam.pos - np.floor(foam.pos + f(0.5))
    pos = torch.as_tensor(np.ascontiguousarray(p, np.float32)).cuda()
    rad = torch.as_tensor(foam.rad).cuda()
    ctx.jfa_run(pos, rad, n)
    torch.cuda.synchronize()
    assert ctx.jfa_stats(n, rad)["finalize_iterations"] >= 2
    # the last block leaves the finalize kernel at its 2nd grid barrier
    ctx.test_barrier_plan(2)
    t0 = time.perf_counter()
    ctx.jfa_run(pos, rad, n)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    assert ctx.device_error() == FOS_E_TIMEOUT
    assert dt < 0.5
    ctx.test_barrier_plan(0)
    ctx.clear_device_error()
    ref = FoamSim(cfg, foam.pos, foam.rad, use_graph=False)
    ref.initialize()
    _frames(ref, 2)
    again = FoamSim(cfg, foam.pos, foam.rad, use_graph=False, ctx=ctx)
    again.initialize()
    _frames(again, 2)
    assert ctx.device_error() == 0
    assert _same_state(again, ref)
    ref.ctx.close()
    ctx.close()
