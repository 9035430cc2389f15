"""fos_grid_build_noalloc: the hash-grid rebuild for callers that cannot
allocate device memory when they need the grid (a host whose own allocator owns
all device memory, a frame loop that cannot afford cudaMalloc's device
synchronisation, a C host without a context).  It must produce exactly what the
context-based fos_grid_build produces, call after call, while its scratch lives
in one static device array that every call reuses.

Collected last on purpose (file name) so that a run stopping at the first
failure has already run every other test; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from fos import _lib, inputs
from fos.config import FosConfig
from fos.context import Context

pytestmark = pytest.mark.gpu

MAX_N = 65536


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _noalloc(pos, n, G, L, cc, cs, ci):
    return _lib.load().fos_grid_build_noalloc(
        _ptr(pos), int(n), int(G), float(L), _ptr(cc), _ptr(cs), _ptr(ci),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))


def _outputs(G3, n):
    z = lambda k: torch.full((k,), -7, dtype=torch.int32, device="cuda")
    return z(G3), z(G3), z(max(n, 1))


def test_noalloc_grid_build_matches_context_build_on_consecutive_calls():
    foam = inputs.headline()
    cfg = FosConfig.for_foam(foam)
    G = cfg.grid_res()
    G3 = G ** 3
    ctx = Context(cfg, max_n=foam.n, max_res=cfg.JFA_RES)
    rng = np.random.default_rng(42)
    # two calls in a row with different inputs and sizes: the second call must
    # not see anything left in the shared scratch by the first
    cases = [(foam.pos, foam.n),
             ((foam.pos[:7001] + rng.uniform(-0.6, 0.6, (7001, 3))).astype(np.float32), 7001)]
    for k, (pos_np, n) in enumerate(cases):
        a = torch.as_tensor(np.ascontiguousarray(pos_np, np.float32)).cuda()
        b = a.clone()
        ra = _outputs(G3, n)
        rb = _outputs(G3, n)
        ctx.grid_build(a, n, *ra)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = _noalloc(b, n, G, cfg.DOMAIN_SIZE, *rb)
        assert rc == 0, _lib.load().fos_last_error()
        torch.cuda.synchronize()
        if k > 0:  # after the first call's one-time address lookup
            assert torch.cuda.mem_get_info()[0] == free0
        for x, y in zip(ra, rb):
            assert torch.equal(x, y)
        assert torch.equal(a, b)  # wrapped positions
        assert int(rb[0].sum()) == n


def test_noalloc_rejects_more_than_its_capacity():
    G = 17
    n = MAX_N + 1
    pos = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    cc, cs, ci = _outputs(G ** 3, n)
    rc = _noalloc(pos, n, G, 1.0, cc, cs, ci)
    assert rc == 2  # FOS_E_CAPACITY
    assert b"FOS_NOALLOC_MAX_PARTICLES" in _lib.load().fos_last_error()
    torch.cuda.synchronize()
    assert int((cc == -7).sum()) == G ** 3  # nothing was launched


@pytest.mark.parametrize("n", [0, MAX_N])
def test_noalloc_edge_sizes_match_context_build(n):
    """n = 0 (only the histogram clear and the scan run) and n at the cap (the
    last scratch entry of the cell half and the first of the rank half), on a
    17^3 grid, against the context build on the same positions."""
    G = 17
    G3 = G ** 3
    cfg = FosConfig(DOMAIN_SIZE=1.0, GRID_RES=G, JFA_RES=32)
    ctx = Context(cfg, max_n=max(n, 1), max_res=32)
    rng = np.random.default_rng(n + 5)
    pos_np = rng.uniform(-0.7, 0.7, (max(n, 1), 3)).astype(np.float32)
    a = torch.as_tensor(pos_np).cuda()
    b = a.clone()
    ra, rb = _outputs(G3, n), _outputs(G3, n)
    ctx.grid_build(a, n, *ra)
    rc = _noalloc(b, n, G, 1.0, *rb)
    assert rc == 0, _lib.load().fos_last_error()
    torch.cuda.synchronize()
    assert torch.equal(ra[0], rb[0]) and torch.equal(ra[1], rb[1])
    assert torch.equal(ra[2][:n], rb[2][:n])
    assert torch.equal(a, b)
    assert int(rb[0].sum()) == n
    if n == 0:
        assert int(rb[0].abs().sum()) == 0 and int(rb[1].abs().sum()) == 0


def test_noalloc_rejects_a_grid_above_its_cap():
    G = 257
    pos = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    cc, cs, ci = _outputs(8, 4)
    rc = _noalloc(pos, 4, G, 1.0, cc, cs, ci)
    assert rc == 1  # FOS_E_ARG
    assert b"grid_res" in _lib.load().fos_last_error()
    torch.cuda.synchronize()
    assert int((cc == -7).sum()) == 8  # nothing was launched
