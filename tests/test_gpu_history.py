"""Rollout history (``lbm_rollout_history`` / ``LBMNode.run_with_history``),
the node's part of ``GraphManager.run_scan_with_history``
(graph_manager.py:2753-2805): record r equals ``run`` with (r + 1) * every
steps, bit for bit, for every field and storage form, and the final state
equals ``run`` with n_steps."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _node(storage, lattice="D3Q19", seed=2):
    from maddening_b200 import LBMNode
    rng = np.random.default_rng(seed)
    grid = (6, 5, 64) if lattice == "D3Q19" else (9, 64)
    D = len(grid)
    wall = rng.random(grid) < 0.1
    wall[0] = wall[-1] = False
    node = LBMNode("h", 1.0, grid_shape=grid, viscosity=0.06, lattice=lattice, wall_mask=wall,
                   storage=storage)
    st = node.initial_state()
    st["f"] = torch.as_tensor(node.lattice.w * (1 + 1e-3 * rng.standard_normal(
        grid + (node.lattice.Q,))), device="cuda").to(st["f"].dtype)
    bi = {"inlet_pressure": np.float32(1 / 3 + 1e-3), "outlet_pressure": np.float32(1 / 3),
          "body_force": rng.uniform(-1e-5, 1e-5, grid + (D,)).astype(np.float32)}
    return node, st, bi


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("n,every", [(7, 1), (9, 3), (10, 4), (1, 1)])
def test_history_records_equal_runs(storage, n, every):
    node, st, bi = _node(storage)
    final, hist = node.run_with_history(st, bi, n, every=every)
    nrec = n // every
    for key in ("f", "density", "velocity", "pressure"):
        assert hist[key].shape[0] == nrec
    for r in range(nrec):
        ref = node.run(st, bi, (r + 1) * every)
        for key in ("f", "density", "velocity", "pressure"):
            assert torch.equal(hist[key][r], ref[key]), (r, key)
    ref = node.run(st, bi, n)
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.equal(final[key], ref[key]), key


def test_history_of_selected_fields_d2q9():
    node, st, bi = _node("f32", "D2Q9")
    final, hist = node.run_with_history(st, bi, 6, every=2, fields=("velocity",))
    assert set(hist) == {"velocity"} and hist["velocity"].shape == (3, 9, 64, 2)
    for r in range(3):
        assert torch.equal(hist["velocity"][r], node.run(st, bi, 2 * (r + 1))["velocity"])
