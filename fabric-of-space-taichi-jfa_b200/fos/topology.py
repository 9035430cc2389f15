"""Drop-in for the reference's topology.py on libfos (fos_topo_*).

Same module fields (``topo_deg``, ``topo_deg_ema``, ``topo_pairs``,
``topo_pair_count``, ``topo_truncated``, allocated by ``allocate_fields``) and
the same functions with the same arguments; CUDA tensors in place of Taichi
fields.  The constants come from the runtime configuration
(``FosConfig.TOPO_*``, ``MAX_TOPO_NEIGHBORS``, ``CELL_SIZE``).  The grid
arguments are the CSR cell arrays of the last rebuild.
"""
from __future__ import annotations

import torch

from . import runtime
from ._lib import call
from .context import ptr, stream

topo_deg = None          # [max_n] int32
topo_deg_ema = None      # [max_n] float32
topo_pairs = None        # [max_n, MAX_TOPO_NEIGHBORS] int32
topo_pair_count = None   # [max_n] int32
topo_truncated = None    # [max_n] int32


def _t(x):
    return getattr(x, "tensor", x)


def allocate_fields(max_n: int):
    """topology.allocate_fields (topology.py:49-62): zeroed fields on the
    runtime context's device."""
    global topo_deg, topo_deg_ema, topo_pairs, topo_pair_count, topo_truncated
    dev = torch.device("cuda", runtime.ctx().device)
    cap = int(runtime.config().MAX_TOPO_NEIGHBORS)
    topo_deg = torch.zeros(max_n, dtype=torch.int32, device=dev)
    topo_deg_ema = torch.zeros(max_n, dtype=torch.float32, device=dev)
    topo_pairs = torch.zeros((max_n, cap), dtype=torch.int32, device=dev)
    topo_pair_count = torch.zeros(max_n, dtype=torch.int32, device=dev)
    topo_truncated = torch.zeros(max_n, dtype=torch.int32, device=dev)


def _grid(cell_start, cell_count, cell_indices):
    return (ptr(_t(cell_start), torch.int32, "cell_start"),
            ptr(_t(cell_count), torch.int32, "cell_count"),
            ptr(_t(cell_indices), torch.int32, "cell_indices"))


def build_topo_candidates(pos, rad, cell_start, cell_count, cell_indices, n: int):
    """topology.build_topo_candidates (topology.py:68-135)."""
    cfg = runtime.config()
    call("fos_topo_candidates", runtime.ctx().h, ptr(_t(pos), torch.float32, "pos"),
         ptr(_t(rad), torch.float32, "rad"), *_grid(cell_start, cell_count, cell_indices), int(n),
         float(cfg.TOPO_MAX_RADIUS_MULTIPLE), int(cfg.MAX_TOPO_NEIGHBORS),
         ptr(topo_pairs, torch.int32, "topo_pairs"),
         ptr(topo_pair_count, torch.int32, "topo_pair_count"),
         ptr(topo_truncated, torch.int32, "topo_truncated"), stream())


def gabriel_test_topological_degree(pos, rad, cell_start, cell_count, cell_indices, n: int,
                                    frame: int):
    """topology.gabriel_test_topological_degree (topology.py:140-262)."""
    cfg = runtime.config()
    call("fos_topo_gabriel", runtime.ctx().h, ptr(_t(pos), torch.float32, "pos"),
         *_grid(cell_start, cell_count, cell_indices), int(n), int(frame), cfg.cell_size(),
         int(cfg.TOPO_PAIR_SUBSAMPLING_STRIDE), int(bool(cfg.TOPO_EARLY_EXIT_HIGH_DEGREE)),
         float(cfg.TOPO_DEG_HIGH), int(cfg.MAX_TOPO_NEIGHBORS),
         ptr(topo_pairs, torch.int32, "topo_pairs"),
         ptr(topo_pair_count, torch.int32, "topo_pair_count"),
         ptr(topo_deg_ema, torch.float32, "topo_deg_ema"), ptr(topo_deg, torch.int32, "topo_deg"),
         stream())


def update_topo_ema(ema_alpha: float, n: int):
    """topology.update_topo_ema (topology.py:265-283)."""
    call("fos_topo_ema", runtime.ctx().h, ptr(topo_deg, torch.int32, "topo_deg"),
         ptr(topo_deg_ema, torch.float32, "topo_deg_ema"), float(ema_alpha), int(n), stream())


def commit_topo_to_ema(alpha: float, n: int):
    """topology.commit_topo_to_ema (topology.py:448-455)."""
    update_topo_ema(alpha, n)


def update_radii_topological(rad, deg_effective, deg_low, deg_high, gain_grow, gain_shrink,
                             r_min, r_max, n: int):
    """topology.update_radii_topological (topology.py:286-322)."""
    call("fos_topo_update_radii", runtime.ctx().h, ptr(_t(rad), torch.float32, "rad"),
         ptr(_t(deg_effective), torch.float32, "deg_effective"), float(deg_low), float(deg_high),
         float(gain_grow), float(gain_shrink), float(r_min), float(r_max), int(n), stream())


def gabriel_update_batched(pos, rad, cell_start, cell_count, cell_indices, n: int,
                           batch_idx: int, num_batches: int, subsample_q: int, frame: int):
    """topology.gabriel_update_batched (topology.py:335-446); adds to topo_deg."""
    cfg = runtime.config()
    call("fos_topo_batched", runtime.ctx().h, ptr(_t(pos), torch.float32, "pos"),
         ptr(_t(rad), torch.float32, "rad"), *_grid(cell_start, cell_count, cell_indices), int(n),
         int(batch_idx), int(num_batches), int(subsample_q), int(frame),
         float(cfg.TOPO_MAX_RADIUS_MULTIPLE), cfg.cell_size(), int(cfg.MAX_TOPO_NEIGHBORS),
         ptr(topo_pairs, torch.int32, "topo_pairs"),
         ptr(topo_pair_count, torch.int32, "topo_pair_count"),
         ptr(topo_truncated, torch.int32, "topo_truncated"), ptr(topo_deg, torch.int32, "topo_deg"),
         stream())


def knn_topo_degree(pos, rad, cell_start, cell_count, cell_indices, n: int, k: int):
    """topology.knn_topo_degree (topology.py:458-505)."""
    cfg = runtime.config()
    call("fos_topo_knn", runtime.ctx().h, ptr(_t(pos), torch.float32, "pos"),
         ptr(_t(rad), torch.float32, "rad"), *_grid(cell_start, cell_count, cell_indices), int(n),
         int(k), float(cfg.TOPO_MAX_RADIUS_MULTIPLE), ptr(topo_deg, torch.int32, "topo_deg"),
         stream())
