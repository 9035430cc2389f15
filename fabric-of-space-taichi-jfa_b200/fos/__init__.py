"""fos -- B200-native hot path of the Fabric-of-Space foam simulator.

Modules mirror the reference's call surface: ``fos.jfa`` (jfa.py),
``fos.grid`` (grid.py), ``fos.dynamics`` (dynamics.py); ``fos.driver`` runs
whole frames in run.py's order.  All device work is libfos.so (hand-written
sm_100a CUDA behind the C ABI in include/fos.h); torch supplies device buffers
and streams only.
"""
from ._lib import FosError  # noqa: F401
from .config import FosConfig  # noqa: F401

__all__ = ["FosError", "FosConfig"]
