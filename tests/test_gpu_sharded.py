"""The slab-sharded runner (``ShardedLBM``) on the GPU: a rollout split into
slabs along axis 0, kept in the kernels' state layout between steps, equals
``LBMNode.run`` on the whole lattice bit for bit (FP32 and FP16 storage) --
with one rank (pads filled locally), run in one call or in pieces, and with
two ranks sharing this GPU over gloo (the crossing populations staged through
host memory between steps; no kernel waits on another rank)."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

GRID = (16, 12, 10)
STEPS = 7


def _setup(storage="f32", grid=GRID):
    from maddening_b200 import LBMNode
    rng = np.random.default_rng(3)
    wall = rng.random(grid) < 0.1
    node = LBMNode("s", 1.0, grid_shape=grid, viscosity=0.06, wall_mask=wall,
                   inlet_face="y_min", outlet_face="y_max", storage=storage)
    st = node.initial_state()
    st["f"] = torch.as_tensor(node.lattice.w * (1 + 1e-3 * rng.standard_normal(grid + (19,))),
                              device="cuda").float()
    bi = {"body_force": np.array([1e-5, -2e-6, 3e-6], dtype=np.float32),
          "inlet_pressure": np.float32(1 / 3 + 1e-3), "outlet_pressure": np.float32(1 / 3)}
    return node, st, bi


def _reference(node, st, bi, steps=STEPS):
    return node.run(st, bi, steps)


@pytest.mark.parametrize("grid", [GRID, (8, 12, 16)])  # rows of 16: the tiled first step
@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_one_rank_equals_whole_lattice_run(storage, grid):
    from maddening_b200.sharded import ShardedLBM
    node, st, bi = _setup(storage, grid)
    sh = ShardedLBM(node)
    sh.scatter(st)
    sh.run(bi, STEPS)
    out, ref = sh.gather(), _reference(node, st, bi)
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.equal(out[key], ref[key]), key


def test_run_in_pieces_equals_one_run():
    from maddening_b200.sharded import ShardedLBM
    node, st, bi = _setup()
    sh = ShardedLBM(node)
    sh.scatter(st)
    sh.run(bi, 1)
    sh.run(bi, 2)
    sh.run(bi, STEPS - 3)
    out, ref = sh.gather(), _reference(node, st, bi)
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.equal(out[key], ref[key]), key
    field = {"body_force": np.random.default_rng(9).uniform(
        -1e-5, 1e-5, GRID + (3,)).astype(np.float32)}
    sh.scatter(st)
    sh.run(field, 4)
    out, ref = sh.gather(), node.run(st, field, 4)
    assert torch.equal(out["f"], ref["f"]) and torch.equal(out["velocity"], ref["velocity"])


def test_faces_on_the_sharded_axis_are_rejected():
    from maddening_b200 import LBMNode
    from maddening_b200.sharded import ShardedLBM
    node = LBMNode("s", 1.0, grid_shape=GRID, viscosity=0.06)  # faces on x
    sh = ShardedLBM(node)
    sh.scatter(node.initial_state())
    with pytest.raises(ValueError, match="sharded axis 0"):
        sh.run({"inlet_pressure": np.float32(0.34)}, 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out, storage):
    import torch.distributed as dist
    from datetime import timedelta
    from maddening_b200.sharded import ShardedLBM
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        node, st, bi = _setup(storage)
        sh = ShardedLBM(node)
        sh.scatter(st)
        sh.run(bi, STEPS)
        got = sh.gather()
        ok = True
        if rank == 0:
            ref = _reference(node, st, bi)
            ok = all(torch.equal(got[k], ref[k]) for k in ("f", "density", "velocity", "pressure"))
        out.put((rank, ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_two_ranks_equal_whole_lattice_run(storage):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, out, storage)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert res == [(0, True), (1, True)]
