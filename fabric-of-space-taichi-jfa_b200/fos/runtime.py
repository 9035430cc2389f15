"""Process-wide default context used by the module-level drop-in API.

The reference's jfa.py keeps its fields as module globals created by
``init_jfa()`` after ``ti.init()``; grid.py and dynamics.py read GRID_RES and
DOMAIN_SIZE from config.py.  Here one ``Context`` plays that role for
``fos.jfa``, ``fos.grid`` and ``fos.dynamics``.
"""
from __future__ import annotations

from .config import FosConfig

_cfg: FosConfig = FosConfig()
_ctx = None


def configure(cfg: FosConfig):
    """Replace the module configuration (the reference's config.py globals)."""
    global _cfg
    _cfg = cfg
    if _ctx is not None and getattr(_ctx, "h", None):
        _ctx.set_params(cfg)


def config() -> FosConfig:
    return _cfg


def init(max_particles: int | None = None, max_res: int | None = None):
    """Create the default context (jfa.init_jfa, jfa.py:120-204)."""
    global _ctx
    from .context import Context
    if _ctx is not None:
        _ctx.close()
        _ctx = None  # a failed create below leaves no closed context installed
    _ctx = Context(_cfg, max_n=max_particles or _cfg.MAX_PARTICLES,
                   max_res=max_res or max(_cfg.JFA_RES_MAX, _cfg.JFA_RES))
    return _ctx


def ctx():
    if _ctx is None:
        return init()
    return _ctx
