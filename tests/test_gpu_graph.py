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
