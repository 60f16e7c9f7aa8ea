"""Wall-mask generators against the reference's voxelizer and the obstacle
workloads' properties (CPU).

* ``voxelize_vessel`` equals the masks that the reference's own
  ``lbm_geometry.py`` produced on four grids / parameter sets
  (tests/golden/geometry_golden.npz, made by tests/golden/make_geometry.py),
  and passes the reference's voxelizer tests (tests/nodes/test_lbm.py:460-492).
* ``random_spheres`` (the benchmark geometry: radii 4-12, 10 % solid, centres
  16 cells off the x faces) is deterministic per seed, reaches its solid
  fraction without overshooting by more than one sphere, keeps the inlet and
  outlet planes free, and wraps spheres periodically across y and z.
"""

import json
import os

import numpy as np
import pytest

from maddening_b200.geometry import random_spheres, voxelize_vessel

HERE = os.path.dirname(os.path.abspath(__file__))
REF_PARAMS = {"parent_radius": 6.0, "daughter_radius": 4.0, "parent_length": 30.0,
              "daughter_length": 25.0, "bifurcation_angle": 30.0}


def _golden_cases():
    g = np.load(os.path.join(HERE, "golden", "geometry_golden.npz"))
    i = 0
    while f"vessel{i}_grid" in g:
        grid = tuple(int(n) for n in g[f"vessel{i}_grid"])
        params = json.loads(bytes(g[f"vessel{i}_params"]).decode())
        mask = np.unpackbits(g[f"vessel{i}_bits"])[:int(np.prod(grid))].reshape(grid)
        yield grid, params, mask.astype(bool)
        i += 1


@pytest.mark.parametrize("case", list(_golden_cases()), ids=lambda c: "x".join(map(str, c[0])))
def test_voxelize_vessel_equals_reference_masks(case):
    grid, params, ref = case
    mask = voxelize_vessel(grid, params)
    assert mask.dtype == np.bool_ and mask.shape == grid
    np.testing.assert_array_equal(mask, ref)


def test_voxelize_vessel_reasonable_fluid_fraction():
    mask = voxelize_vessel((64, 32, 32), REF_PARAMS)
    fluid = float(np.sum(~mask)) / mask.size
    assert 0.05 < fluid < 0.50


def test_voxelize_vessel_parent_centre_is_fluid():
    mask = voxelize_vessel((64, 32, 32), REF_PARAMS)
    assert not bool(mask[15, 15, 15])


def test_random_spheres_deterministic_per_seed():
    a = random_spheres((64, 48, 40), seed=3)
    b = random_spheres((64, 48, 40), seed=3)
    c = random_spheres((64, 48, 40), seed=4)
    np.testing.assert_array_equal(a, b)
    assert (a != c).any()


@pytest.mark.parametrize("grid", [(64, 64, 64), (96, 80, 72), (256, 64, 64), (128, 128)])
def test_random_spheres_solid_fraction(grid):
    wall = random_spheres(grid, seed=0)
    frac = wall.mean()
    # stops at the first sphere that reaches 10 %: at most one sphere over
    r_max = 12.0
    one = (4 / 3 * np.pi * r_max ** 3 if len(grid) == 3 else np.pi * r_max ** 2) / wall.size
    assert 0.10 <= frac <= 0.10 + one, frac


def test_random_spheres_keeps_inlet_and_outlet_free():
    # centres at x in [16, n - 17] and radii < 12: planes x < 4 and x > n - 5 stay fluid
    wall = random_spheres((96, 64, 64), seed=1)
    assert not wall[:4].any() and not wall[-4:].any()


def test_random_spheres_are_periodic_in_y_and_z():
    """Every sphere is a set of cells within its radius of the centre, with the
    distance taken periodically across y and z: each solid cell lies within
    r_max of a solid cell on the far side when it touches a boundary plane."""
    wall = random_spheres((64, 40, 40), seed=2)
    for a in (1, 2):
        first = np.take(wall, 0, axis=a)
        last = np.take(wall, -1, axis=a)
        if first.any() or last.any():
            # a sphere cut by the boundary continues on the other side
            assert (first & last).any()
