"""B200-native (sm_100a) lattice-Boltzmann node step for MADDENING graphs.

Public API:
    LBMNode                 -- drop-in node (lbm.py:531-1036 contract)
    LatticeDescriptor, d3q19, d2q9
    build()                 -- compile liblbm_b200.so in-tree
"""

from .lattice import LatticeDescriptor, d2q9, d3q19  # noqa: F401
from .build import build  # noqa: F401


def __getattr__(name):
    # torch-dependent pieces load lazily so `build` works without importing torch
    if name == "LBMNode":
        from .node import LBMNode
        return LBMNode
    raise AttributeError(name)
