"""Batched uneven ensemble (``LBMEnsemble`` / ``lbm_batch_rollout``).

Every member of a batched rollout must equal its own ``LBMNode.run`` (the
same arithmetic, so bit for bit), for every launch configuration the
autotuner may pick; one member is also checked against the FP64 oracle.
"""

import numpy as np
import pytest
import torch

from oracle import lbm_ref as R

pytestmark = pytest.mark.gpu


def _members(storage="f32", lattice="D3Q19"):
    from maddening_b200 import LBMNode
    rng = np.random.default_rng(21)
    if lattice == "D3Q19":
        shapes = [(9, 7, 13), (16, 16, 16), (5, 12, 33), (20, 8, 6), (3, 4, 130), (11, 10, 9),
                  (4, 6, 15)]
    else:
        shapes = [(17, 9), (40, 33), (6, 131), (25, 4), (12, 12), (7, 13)]
    nodes, bis, states = [], [], []
    for i, shape in enumerate(shapes):
        tau = float(rng.uniform(0.55, 1.5))
        wall = rng.random(shape) < 0.1
        kw = {}
        bi = {"body_force": rng.uniform(-1e-5, 1e-5, len(shape)).astype(np.float32)}
        if i == 1:
            kw = dict(inlet_face="x_min", outlet_face="x_max")
            wall[0] = wall[-1] = False
            bi["inlet_pressure"] = np.float32(1.0 / 3.0 + 1e-3)
            bi["outlet_pressure"] = np.float32(1.0 / 3.0)
        if i == 2:
            kw = dict(outlet_condition="zero_gradient")
            wall[0] = wall[-1] = False
            bi = {"inlet_velocity": np.array([0.03] + [0.0] * (len(shape) - 1))}
        if i == 3:
            bi["body_force"] = rng.uniform(-1e-5, 1e-5, shape + (len(shape),)).astype(np.float32)
        if i == len(shapes) - 1:
            # faces on the contiguous axis of an odd row (padded state rows)
            ax = "z" if len(shape) == 3 else "y"
            kw = dict(inlet_face=f"{ax}_min", outlet_face=f"{ax}_max",
                      outlet_condition="zero_gradient")
            wall[..., 0] = wall[..., -1] = False
            bi = {"inlet_velocity": np.array([0.0] * (len(shape) - 1) + [0.02]),
                  "body_force": rng.uniform(-1e-5, 1e-5, shape + (len(shape),)).astype(np.float32)}
        node = LBMNode(f"m{i}", 1.0, grid_shape=shape, viscosity=(tau - 0.5) / 3.0,
                       lattice=lattice, wall_mask=wall, storage=storage, **kw)
        st = node.initial_state()
        lat = node.lattice
        f0 = lat.w * (1 + 1e-3 * rng.standard_normal(shape + (lat.Q,)))
        st["f"] = torch.as_tensor(f0, device="cuda").to(st["f"].dtype)
        nodes.append(node)
        bis.append(bi)
        states.append(st)
    return nodes, bis, states


CONFIGS = [{"blocks_per_sm": b, "tile_order": o, "use_graph": g, "group_mib": m}
           for b, o, g, m in ((0, 0, 0, 0), (8, 0, 1, 0), (4, 1, 0, 0), (16, 1, 1, 0),
                              (1, 0, 1, 0), (8, 2, 1, 1), (0, 0, 0, 1), (4, 2, 0, 4096),
                              (0, 2, 1, 0))]


@pytest.mark.parametrize("lattice", ["D3Q19", "D2Q9"])
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f64"])
def test_batched_members_equal_their_own_rollouts(lattice, storage):
    from maddening_b200.batched import LBMEnsemble
    nodes, bis, states = _members(storage, lattice)
    steps = 7
    ref = [n.run(s, b, steps) for n, s, b in zip(nodes, states, bis)]
    ens = LBMEnsemble(nodes)
    for cfg in CONFIGS:
        out = ens.run(states, bis, steps, cfg)
        for i, (o, r) in enumerate(zip(out, ref)):
            for key in ("f", "density", "velocity", "pressure"):
                assert torch.equal(o[key], r[key]), (cfg, i, key)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_uniform_class_ensemble_equals_own_rollouts(storage):
    """Members that all share one face / force form run the compile-time
    specialised batched kernel."""
    from maddening_b200.batched import LBMEnsemble, uneven_ensemble
    nodes, bis = uneven_ensemble(5, seed=3, lo=8, hi=40, storage=storage, device="cuda")
    states = [n.initial_state() for n in nodes]
    ref = [n.run(s, b, 6) for n, s, b in zip(nodes, states, bis)]
    ens = LBMEnsemble(nodes)
    for cfg in CONFIGS[:3]:
        out = ens.run(states, bis, 6, cfg)
        for i, (o, r) in enumerate(zip(out, ref)):
            for key in ("f", "density", "velocity", "pressure"):
                assert torch.equal(o[key], r[key]), (cfg, i, key)


def test_grouped_launch_rejects_round_robin_order():
    from maddening_b200 import _lib
    from maddening_b200.batched import LBMEnsemble
    nodes, bis, states = _members()
    ens = LBMEnsemble(nodes)
    with pytest.raises(_lib.LbmError, match="instance-major"):
        ens.run(states, bis, 2, {"blocks_per_sm": 0, "tile_order": 1, "use_graph": 0,
                                 "group_mib": 8})


def test_batched_member_matches_fp64_oracle():
    from maddening_b200.batched import LBMEnsemble
    nodes, bis, states = _members("f64")
    ens = LBMEnsemble(nodes)
    out = ens.run(states, bis, 5)
    i = 0
    node = nodes[i]
    orc = R.OracleLBM(node._grid_shape, node.viscosity, "D3Q19", wall_mask=node._wall_np)
    so = orc.initial_state()
    so["f"] = states[i]["f"].cpu().numpy()
    so = orc.run(so, bis[i], 5)
    np.testing.assert_allclose(out[i]["f"].cpu().numpy(), so["f"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(out[i]["velocity"].cpu().numpy(), so["velocity"], rtol=0, atol=1e-14)


def test_autotune_picks_a_valid_config():
    from maddening_b200.batched import LBMEnsemble
    nodes, bis, states = _members()
    ens = LBMEnsemble(nodes)
    cfg = ens.autotune(states, bis, n_steps=4, use_cache=False)
    assert set(cfg) == {"blocks_per_sm", "tile_order", "use_graph", "group_mib"}
    assert cfg["blocks_per_sm"] in (0, 4, 8, 16) and cfg["tile_order"] in (0, 1, 2)
    assert cfg["use_graph"] in (0, 1) and cfg["group_mib"] >= 0
    ref = [n.run(s, b, 3) for n, s, b in zip(nodes, states, bis)]
    out = ens.run(states, bis, 3)
    for o, r in zip(out, ref):
        assert torch.equal(o["f"], r["f"])
