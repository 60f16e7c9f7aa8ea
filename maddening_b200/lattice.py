"""Lattice descriptors with the reference's names and direction order.

``LatticeDescriptor``, ``d3q19()`` and ``d2q9()`` mirror
``src/maddening/nodes/lbm.py:57-173`` (NumPy arrays so they stay concrete
inside traced code).  The CUDA kernels carry the same constants at compile
time (``csrc/lbm_lattice.cuh``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class LatticeDescriptor:
    name: str
    e: np.ndarray    # (Q, D) int32
    w: np.ndarray    # (Q,) float64
    opp: np.ndarray  # (Q,) int32
    cs2: float
    D: int
    Q: int


def _opposites(e: np.ndarray) -> np.ndarray:
    q = e.shape[0]
    return np.array([next(p for p in range(q) if np.array_equal(e[p], -e[i]))
                     for i in range(q)], dtype=np.int32)


def d3q19() -> LatticeDescriptor:
    """D3Q19: rest, 6 axis neighbours, 12 edge neighbours (xy, xz, yz pairs)."""
    axes = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    edges = []
    for a, b in ((0, 1), (0, 2), (1, 2)):
        for sb in (1, -1):
            for sa in (1, -1):
                v = [0, 0, 0]
                v[a], v[b] = sa, sb
                edges.append(tuple(v))
    e = np.array([(0, 0, 0)] + axes + edges, dtype=np.int32)
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float64)
    return LatticeDescriptor("D3Q19", e, w, _opposites(e), 1.0 / 3.0, 3, 19)


def d2q9() -> LatticeDescriptor:
    """D2Q9: rest, 4 axis neighbours, 4 diagonals."""
    e = np.array([(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1),
                  (1, 1), (-1, 1), (1, -1), (-1, -1)], dtype=np.int32)
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, dtype=np.float64)
    return LatticeDescriptor("D2Q9", e, w, _opposites(e), 1.0 / 3.0, 2, 9)


def by_name(name: str) -> LatticeDescriptor:
    if name.upper() == "D3Q19":
        return d3q19()
    if name.upper() == "D2Q9":
        return d2q9()
    raise ValueError(f"Unknown lattice '{name}'. Supported: 'D3Q19', 'D2Q9'.")
