"""GPU parity of the periodic hash grid (counting sort) against the oracle.

Bar: cell_count, cell_start, cell_indices (ascending inside each cell) and the
wrapped positions are bit-exact.
"""
import numpy as np
import pytest
import torch

from fos import inputs
from fos.config import FosConfig
from fos.context import Context
from oracle import oracle as O

from helpers import oracle_params

pytestmark = pytest.mark.gpu


def _setup(foam):
    cfg = FosConfig.for_foam(foam)
    ctx = Context(cfg, max_n=foam.n, max_res=cfg.JFA_RES)
    G3 = cfg.grid_res() ** 3
    z = lambda k: torch.zeros(k, dtype=torch.int32, device="cuda")
    return cfg, ctx, z(G3), z(G3), z(G3), z(foam.n)


@pytest.mark.parametrize("name", ["small", "headline", "stress"])
def test_fused_grid_build_bit_exact(name):
    foam = {"small": inputs.small, "headline": inputs.headline, "stress": inputs.stress}[name]()
    p = oracle_params(foam)
    pos_o = np.ascontiguousarray(foam.pos, np.float32).copy()  # unwrapped [0,1)^3 input
    cc, cs, ci = O.grid_build(pos_o, p)
    cfg, ctx, gcc, gcs, gcw, gci = _setup(foam)
    assert cfg.grid_res() == p.G
    pos = torch.as_tensor(np.ascontiguousarray(foam.pos, np.float32)).cuda()
    ctx.grid_build(pos, foam.n, gcc, gcs, gci)
    torch.cuda.synchronize()
    assert np.array_equal(gcc.cpu().numpy(), cc)
    assert np.array_equal(gcs.cpu().numpy(), cs)
    assert np.array_equal(gci.cpu().numpy(), ci)
    assert np.array_equal(pos.cpu().numpy(), pos_o)
    assert int(gcc.sum()) == foam.n  # CSR integrity check (run.py:486-500)


def test_reference_call_sequence():
    """clear_grid, count, prefix_sum, copy_cell_pointers, scatter (run.py:476-504)."""
    foam = inputs.headline()
    p = oracle_params(foam)
    pos_o = np.ascontiguousarray(foam.pos, np.float32).copy()
    cc, cs, ci = O.grid_build(pos_o, p)
    cfg, ctx, gcc, gcs, gcw, gci = _setup(foam)
    pos = torch.as_tensor(np.ascontiguousarray(foam.pos, np.float32)).cuda()
    ctx.grid_clear(gcc)
    ctx.grid_count(pos, gcc, foam.n)
    ctx.grid_prefix_sum(gcc, gcs)
    ctx.grid_copy_pointers(gcs, gcw)
    ctx.grid_scatter(pos, gcw, gci, foam.n)
    torch.cuda.synchronize()
    assert np.array_equal(gcc.cpu().numpy(), cc)
    assert np.array_equal(gcs.cpu().numpy(), cs)
    assert np.array_equal(gci.cpu().numpy(), ci)
    assert np.array_equal(gcw.cpu().numpy(), cs + cc)
    assert np.array_equal(pos.cpu().numpy(), pos_o)


def test_crowded_cells_and_boundaries():
    """Many particles in one cell, particles exactly on faces and at +-L/2."""
    n = 3000
    rng = np.random.default_rng(4)
    pos = np.empty((n, 3), np.float32)
    pos[:1000] = 0.01 * rng.random((1000, 3), dtype=np.float32)
    pos[1000:2000] = rng.choice(np.array([-0.5, 0.5, 0.0, 1.0 / 17, -1.0 / 17], np.float32),
                                (1000, 3))
    pos[2000:] = rng.uniform(-2, 2, (1000, 3)).astype(np.float32)
    from fos.inputs import Foam
    foam = Foam("crowd", pos, np.full(n, 0.01, np.float32), 64, 0.01, 0.03, 10, 16, 4, 10, 1, 1,
                1, 0)
    p = oracle_params(foam)
    pos_o = pos.copy()
    cc, cs, ci = O.grid_build(pos_o, p)
    cfg, ctx, gcc, gcs, gcw, gci = _setup(foam)
    t = torch.as_tensor(pos).cuda()
    ctx.grid_build(t, n, gcc, gcs, gci)
    torch.cuda.synchronize()
    assert np.array_equal(gcc.cpu().numpy(), cc)
    assert np.array_equal(gci.cpu().numpy(), ci)
    assert np.array_equal(t.cpu().numpy(), pos_o)
