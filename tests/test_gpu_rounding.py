"""Stochastic rounding of the 16-bit state, end to end: in a periodic box
(no walls) a uniform force F raises the total momentum sum(f e) by exactly
N F per step.  The per-step gain of an offset (~3 g = 6e-6) is below an FP16
unit of the offsets it is added to (up to ~1e-2), so round-to-nearest storage
distorts the growth (+17 % after 2000 steps in the FP64 oracle with its offsets
rounded to FP16 on an 8^3 box); with stochastic rounding the total stays within
noise of N F n (3e-5 in the same emulation)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_momentum_growth_under_a_small_force(storage):
    from maddening_b200 import LBMNode
    grid, steps = (32, 32, 32), 2000
    F = np.array([2e-6, 0.0, 0.0], dtype=np.float32)
    node = LBMNode("r", 1.0, grid_shape=grid, viscosity=0.1, storage=storage)
    st = node.initial_state()
    j0 = node.mass_momentum(st["f"])[1:].cpu().numpy()
    out = node.run(st, {"body_force": F}, steps)
    j1 = node.mass_momentum(out["f"])[1:].cpu().numpy()
    expect = steps * np.prod(grid) * F.astype(np.float64)
    assert abs((j1 - j0)[0] - expect[0]) <= 1e-3 * expect[0], (j1 - j0, expect)


@pytest.mark.parametrize("storage,tol", [("f16", 1e-3), ("bf16", 3e-3)])
def test_momentum_keeps_growing_over_5000_steps(storage, tol):
    """The rounding bits are a function of the cell's index and state, with no
    step counter, so each step is a fixed map of the stored state: a run could
    only stall if every stored value rounded back to itself.  Under a force
    whose per-step gain of an offset (3 F = 1.5e-6) is about one FP16 unit,
    the total momentum still follows N F n at the midpoint and after 5000
    steps."""
    from maddening_b200 import LBMNode
    grid = (32, 32, 32)
    F = np.array([5e-7, 0.0, 0.0], dtype=np.float32)
    node = LBMNode("r", 1.0, grid_shape=grid, viscosity=0.1, storage=storage)
    st = node.initial_state()
    j0 = node.mass_momentum(st["f"])[1].item()
    for n in (2500, 5000):
        st = node.run(st, {"body_force": F}, 2500)
        j = node.mass_momentum(st["f"])[1].item()
        expect = n * np.prod(grid) * float(F[0])
        assert abs((j - j0) - expect) <= tol * expect, (n, j - j0, expect)
