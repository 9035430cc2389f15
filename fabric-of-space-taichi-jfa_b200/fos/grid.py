"""Drop-in for the reference's grid.py kernels (grid.py:145-309) on libfos.

Arguments are CUDA tensors: pos [>=n, 3] float32, cell arrays [GRID_RES^3]
int32, cell_indices [>=n] int32.  GRID_RES and DOMAIN_SIZE come from the
module configuration (fos.runtime.config()).  scatter_particles leaves each
cell's slice of cell_indices ascending (the serial order).
"""
from __future__ import annotations

from . import runtime


def _c():
    return runtime.ctx()


def grid_res() -> int:
    return runtime.config().grid_res()


def clear_grid(cell_count):
    """grid.clear_grid (grid.py:145-155)."""
    _c().grid_clear(cell_count)


def count_particles_per_cell(pos, cell_count, n: int):
    """grid.count_particles_per_cell (grid.py:186-222)."""
    _c().grid_count(pos, cell_count, n)


def prefix_sum(cell_count, cell_start):
    """grid.prefix_sum (grid.py:229-243): exclusive scan."""
    _c().grid_prefix_sum(cell_count, cell_start)


def copy_cell_pointers(cell_start, cell_write):
    """grid.copy_cell_pointers (grid.py:250-261)."""
    _c().grid_copy_pointers(cell_start, cell_write)


def scatter_particles(pos, cell_write, cell_indices, n: int):
    """grid.scatter_particles (grid.py:268-309): wraps pos in place."""
    _c().grid_scatter(pos, cell_write, cell_indices, n)


def rebuild_grid(pos, n: int, cell_count, cell_start, cell_indices):
    """rebuild_grid (run.py:476-504) as one fused call."""
    _c().grid_build(pos, n, cell_count, cell_start, cell_indices)
