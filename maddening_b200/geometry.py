"""Wall-mask generators (True = wall), the convention of
``src/maddening/nodes/lbm_geometry.py``.

* ``voxelize_vessel`` -- Y-bifurcation vessel with the reference's parameters
  and semantics (``lbm_geometry.py:17-142``): a cell is fluid when its
  distance to the parent or to either daughter centre-line segment is below
  that segment's radius.
* ``random_spheres`` -- seeded sphere obstacles for the obstacle-flow
  workloads: centres uniform in the box (kept ``margin`` cells away from the
  first and last plane of axis 0, the inlet/outlet axis), radii uniform in
  [r_min, r_max], periodic in the other axes, added one at a time until the
  solid fraction reaches ``solid_fraction``.
* ``z_walls`` -- walls on the first and last plane of the last axis (the
  channel workloads).
"""

from __future__ import annotations

import numpy as np


def _segment_distance(pts, a, b):
    ab = b - a
    ll = float(ab @ ab)
    t = np.clip(((pts - a) @ ab) / max(ll, 1e-10), 0.0, 1.0)
    closest = a + t[..., None] * ab
    return np.sqrt(np.sum((pts - closest) ** 2, axis=-1))


def voxelize_vessel(grid_shape: tuple, vessel_params: dict) -> np.ndarray:
    nx, ny, nz = grid_shape
    pr = vessel_params["parent_radius"]
    dr = vessel_params["daughter_radius"]
    pl = vessel_params["parent_length"]
    dl = vessel_params["daughter_length"]
    ang = np.deg2rad(vessel_params["bifurcation_angle"])
    mid = np.array([0.0, (ny - 1) / 2.0, (nz - 1) / 2.0])
    pts = np.stack(np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64),
                               np.arange(nz, dtype=np.float64), indexing="ij"), axis=-1)
    start = mid.copy()
    bif = mid + np.array([pl, 0.0, 0.0])
    fluid = _segment_distance(pts, start, bif) < pr
    for s in (-1.0, 1.0):
        d = np.array([np.cos(ang), s * np.sin(ang), 0.0])
        fluid |= _segment_distance(pts, bif, bif + dl * d) < dr
    return ~fluid


def random_spheres(grid_shape, seed: int = 0, r_min: float = 4.0, r_max: float = 12.0,
                   solid_fraction: float = 0.10, margin: int = 16,
                   max_spheres: int = 1_000_000) -> np.ndarray:
    shape = tuple(int(n) for n in grid_shape)
    D = len(shape)
    rng = np.random.default_rng(seed)
    wall = np.zeros(shape, dtype=bool)
    total = wall.size
    solid = 0
    lo0 = float(margin)
    hi0 = float(shape[0] - 1 - margin)
    if hi0 < lo0:
        lo0, hi0 = 0.0, float(shape[0] - 1)
    for _ in range(max_spheres):
        if solid >= solid_fraction * total:
            break
        c = np.empty(D)
        c[0] = rng.uniform(lo0, hi0)
        for a in range(1, D):
            c[a] = rng.uniform(0.0, shape[a])
        r = rng.uniform(r_min, r_max)
        # bounding box, axis 0 clipped (non-periodic), others wrapped
        idx = []
        for a in range(D):
            lo = int(np.floor(c[a] - r))
            hi = int(np.ceil(c[a] + r))
            if a == 0:
                idx.append(np.arange(max(lo, 0), min(hi, shape[0] - 1) + 1))
            else:
                idx.append(np.arange(lo, hi + 1))
        grids = np.meshgrid(*idx, indexing="ij")
        d2 = sum((g - c[a]) ** 2 for a, g in enumerate(grids))
        inside = d2 < r * r
        cells = tuple(g[inside] % shape[a] if a > 0 else g[inside] for a, g in enumerate(grids))
        flat = np.unique(np.ravel_multi_index(cells, shape))
        view = wall.reshape(-1)
        solid += int(np.count_nonzero(~view[flat]))
        view[flat] = True
    return wall


def z_walls(grid_shape) -> np.ndarray:
    """Walls on the first and last plane of the last axis (True = wall)."""
    wall = np.zeros(tuple(int(n) for n in grid_shape), dtype=bool)
    wall[..., 0] = True
    wall[..., -1] = True
    return wall
