"""Drop-in for the reference's jfa.py call surface on libfos.

Same names, argument order and return values as jfa.py (cited per function);
fields are torch tensors on the GPU wrapped in ``Field`` so that run.py-style
code (``jfa.fsc.to_numpy()``, ``jfa.fsc[0]``, ``jfa.power_beta_current[None]``)
keeps working.  ``pos``/``rad`` arguments are CUDA tensors ([>=n, 3] and
[>=n] float32) in place of Taichi fields.
"""
from __future__ import annotations

import numpy as np
import torch

from . import runtime
from ._lib import MAX_NEIGHBORS as _S

MAX_NEIGHBORS = _S                # jfa.py:74
MAX_PARTICLES = 50000             # jfa.py:67
EXPECTED_FACE_SCALE = 1.5         # jfa.py:58
T_ADD = 0.15                      # jfa.py:63
T_DROP = 0.10                     # jfa.py:64
JFA_RES = 128                     # jfa.py:80
JFA_NUM_PASSES = 8                # jfa.py:83
VOXEL_SIZE = runtime.config().DOMAIN_SIZE / JFA_RES
tiles_per_axis = 0                # jfa.py:117

fsc = fsc_ema = face_ids = face_counts = neighbor_list = None
neighbor_count = neighbor_used_count = neighbor_prev_scores = None
power_beta_current = None
tile_dirty = pos_prev = rad_prev = None
_tile_store = None


class Field:
    """Minimal Taichi-field look-alike over a torch CUDA tensor."""

    def __init__(self, tensor: torch.Tensor):
        self.tensor = tensor

    @property
    def shape(self):
        return tuple(self.tensor.shape)

    def to_numpy(self) -> np.ndarray:
        return self.tensor.detach().cpu().numpy()

    def from_numpy(self, a):
        self.tensor.copy_(torch.as_tensor(a, dtype=self.tensor.dtype))

    def fill(self, v):
        self.tensor.fill_(v)

    def __getitem__(self, idx):
        v = self.tensor[idx]
        return v.item() if v.numel() == 1 else v

    def __setitem__(self, idx, value):
        self.tensor[idx] = value


class _PowerBeta:
    """power_beta_current (jfa.py:184): a 0-d field; writes go to the context."""

    def __getitem__(self, idx):
        return float(runtime.config().POWER_BETA)

    def __setitem__(self, idx, value):
        cfg = runtime.config()
        if float(value) != cfg.POWER_BETA:
            cfg.POWER_BETA = float(value)
            runtime.ctx().set_params(cfg)


def _tensor(x):
    return x.tensor if isinstance(x, Field) else x


def init_jfa(max_particles: int | None = None, max_res: int | None = None):
    """jfa.init_jfa (jfa.py:120-204): allocate every field at capacity."""
    global fsc, fsc_ema, face_ids, face_counts, neighbor_list, neighbor_count
    global neighbor_used_count, neighbor_prev_scores, power_beta_current, tiles_per_axis
    global tile_dirty, pos_prev, rad_prev
    cfg = runtime.config()
    ctx = runtime.init(max_particles or cfg.MAX_PARTICLES, max_res)
    fsc = Field(ctx.fsc)
    fsc_ema = Field(ctx.fsc_ema)
    face_ids = Field(ctx.face_ids)
    face_counts = Field(ctx.face_counts)
    neighbor_list = Field(ctx.neighbor_list)
    neighbor_used_count = Field(ctx.neighbor_used_count)
    neighbor_count = neighbor_used_count
    neighbor_prev_scores = Field(ctx.neighbor_prev_scores)
    power_beta_current = _PowerBeta()
    global _tile_store
    max_tiles = (ctx.max_res + 15) // 16
    _tile_store = torch.zeros(max_tiles ** 3, dtype=torch.uint8, device="cuda")
    tile_dirty = Field(_tile_store[:1].view(1, 1, 1))
    pos_prev = Field(torch.zeros((ctx.max_n, 3), dtype=torch.float32, device="cuda"))
    rad_prev = Field(torch.zeros((ctx.max_n,), dtype=torch.float32, device="cuda"))
    set_resolution(cfg.JFA_RES)


def set_resolution(new_res: int):
    """jfa.set_resolution (jfa.py:207-227): clamp to [JFA_RES_MIN, JFA_RES_MAX],
    VOXEL_SIZE = L / R, JFA_NUM_PASSES = ceil(log2 R) + 1."""
    global JFA_RES, VOXEL_SIZE, JFA_NUM_PASSES, tiles_per_axis
    cfg = runtime.config()
    res = max(cfg.JFA_RES_MIN, min(int(new_res), cfg.JFA_RES_MAX))
    ctx = runtime.ctx()
    ctx.set_resolution(res)
    JFA_RES = ctx.res
    VOXEL_SIZE = cfg.DOMAIN_SIZE / JFA_RES
    JFA_NUM_PASSES = ctx.num_passes
    tiles_per_axis = (JFA_RES + 15) // 16  # JFA_TILE_SIZE = 16 (config.py:182)
    if tile_dirty is not None:
        # [t, t, t] view of the contiguous first t^3 bytes (fos_dirty_* layout)
        t = tiles_per_axis
        tile_dirty.tensor = _tile_store[: t ** 3].view(t, t, t)


def run_jfa(pos, rad, active_n: int):
    """jfa.run_jfa (jfa.py:1056-1197): JFA + FSC extraction on the GPU.

    Returns (fsc as numpy [active_n], stats dict with the reference's keys).
    """
    ctx = runtime.ctx()
    ctx.jfa_run(_tensor(pos), _tensor(rad), int(active_n))
    stats = ctx.jfa_stats(int(active_n), _tensor(rad))
    n = int(active_n)
    stats["fsc_ema"] = ctx.fsc_ema[:n].cpu().numpy()
    return ctx.fsc[:n].cpu().numpy(), stats


def validate_jfa(active_n: int) -> dict:
    """jfa.validate_jfa (jfa.py:1400-1426)."""
    return runtime.ctx().validate(int(active_n))


# ---------------------------------------------------------------- dirty tiles
# Instrumentation only in the reference (jfa.py:966-1049; run.py:1021-1047):
# it never changes JFA output.
def mark_dirty_tiles(pos, rad, n: int):
    """jfa.mark_dirty_tiles (jfa.py:966-1008) on libfos (fos_dirty_mark)."""
    from ._lib import call
    from .context import ptr, stream
    cfg = runtime.config()
    call("fos_dirty_mark", runtime.ctx().h, ptr(_tensor(pos), torch.float32, "pos"),
         ptr(_tensor(rad), torch.float32, "rad"), ptr(pos_prev.tensor, torch.float32, "pos_prev"),
         ptr(rad_prev.tensor, torch.float32, "rad_prev"), int(n),
         float(cfg.JFA_DIRTY_POS_THRESHOLD), float(cfg.JFA_DIRTY_RAD_THRESHOLD),
         int(cfg.JFA_DIRTY_HALO), ptr(tile_dirty.tensor, torch.uint8, "tile_dirty"), stream())


def count_dirty_tiles() -> int:
    """jfa.count_dirty_tiles (jfa.py:1011-1024) on libfos (fos_dirty_count)."""
    import ctypes as C
    from ._lib import call
    from .context import ptr, stream
    out = C.c_int()
    call("fos_dirty_count", runtime.ctx().h, ptr(tile_dirty.tensor, torch.uint8, "tile_dirty"),
         C.byref(out), stream())
    return int(out.value)


def clear_dirty_tiles():
    """jfa.clear_dirty_tiles (jfa.py:1027-1034)."""
    tile_dirty.tensor.zero_()


def update_tile_cache(pos, rad, n: int):
    """jfa.update_tile_cache (jfa.py:1037-1049)."""
    pos_prev.tensor[:n] = _tensor(pos)[:n]
    rad_prev.tensor[:n] = _tensor(rad)[:n]


def print_jfa_config():
    """jfa.print_jfa_config: prints the active JFA settings."""
    cfg = runtime.config()
    print(f"[JFA] res={JFA_RES}^3 passes={JFA_NUM_PASSES} voxel={VOXEL_SIZE:.6f} "
          f"beta={cfg.POWER_BETA} early_exit={cfg.JFA_EARLY_EXIT_ENABLED} "
          f"T_ADD={T_ADD} T_DROP={T_DROP} max_neighbors={MAX_NEIGHBORS} (B200 libfos)")
