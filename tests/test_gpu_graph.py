"""LBMNode.run can be captured in a CUDA graph (no host synchronisation or
device allocation outside the graph's memory pool inside run): replaying the
graph gives the plain rollout's bytes, replay after replay."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_captured_rollout_equals_plain(storage):
    from maddening_b200 import LBMNode
    grid = (24, 20, 32)
    wall = np.zeros(grid, dtype=bool)
    wall[:, :, 0] = wall[:, :, -1] = True
    node = LBMNode("g", 1.0, grid_shape=grid, viscosity=0.1, wall_mask=wall, storage=storage)
    bi = {"body_force": np.array([1e-5, 0.0, 0.0], dtype=np.float32)}
    st = node.initial_state()
    ref = node.run(st, bi, 40)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        node.run(st, bi, 40)  # warm-up outside the capture
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out = node.run(st, bi, 40)
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        for key in ("f", "density", "velocity", "pressure"):
            assert torch.equal(out[key], ref[key]), key


@pytest.mark.parametrize("storage,one_pass", [("f32", None), ("f16", None), ("f16", False)])
def test_captured_update_calls_equal_plain(storage, one_pass):
    """Three chained ``update`` calls (the call a graph manager makes each
    step: the one-pass kernel, or the two passes on request) captured once
    and replayed give the plain calls' bytes."""
    from maddening_b200 import LBMNode
    grid = (20, 16, 36)
    rng = np.random.default_rng(2)
    node = LBMNode("u", 1.0, grid_shape=grid, viscosity=0.05, wall_mask=rng.random(grid) < 0.1,
                   outlet_condition="zero_gradient", storage=storage, one_pass=one_pass)
    bi = {"inlet_velocity": np.array([0.04, 0.0, 0.0], dtype=np.float32)}
    st = node.initial_state()

    def three(s):
        for _ in range(3):
            s = node.update(s, bi, 1.0)
        return s

    ref = three(st)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        three(st)
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out = three(st)
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        for key in ("f", "density", "velocity", "pressure"):
            assert torch.equal(out[key], ref[key]), key
