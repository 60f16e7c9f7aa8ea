"""Row-staged state step (bulk copies into shared memory, opt-in with
``staged_rows=True``): bit-identical to the global-memory gather, and its
bounded waits never time out.

The staged kernel serves rollouts whose rows are at least 128 cells long and
a multiple of 16 bytes; the batched ensemble always uses the global-memory
gather, so a one-member ensemble is the reference path.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from oracle import lbm_ref as R

pytestmark = pytest.mark.gpu


def _node(shape, storage, lattice, kind, seed=0):
    from maddening_b200 import LBMNode
    rng = np.random.default_rng(seed)
    wall = rng.random(shape) < 0.08
    kw, bi = {}, {}
    D = len(shape)
    if kind == "faces":
        wall[0] = wall[-1] = False
        kw = dict(outlet_condition="zero_gradient")
        bi = {"inlet_velocity": np.array([0.04] + [0.0] * (D - 1))}
    elif kind == "pressure":
        wall[0] = wall[-1] = False
        bi = {"inlet_pressure": np.float32(1 / 3 + 1e-3), "outlet_pressure": np.float32(1 / 3),
              "body_force": rng.uniform(-1e-5, 1e-5, shape + (D,)).astype(np.float32)}
    else:
        bi = {"body_force": np.array([1e-5, -2e-6, 3e-6][:D], dtype=np.float32)}
    node = LBMNode("s", 1.0, grid_shape=shape, viscosity=0.05, lattice=lattice, wall_mask=wall,
                   storage=storage, staged_rows=True, **kw)
    st = node.initial_state()
    lat = node.lattice
    st["f"] = torch.as_tensor(lat.w * (1 + 1e-3 * rng.standard_normal(shape + (lat.Q,))),
                              device="cuda").to(st["f"].dtype)
    return node, st, bi


@pytest.mark.parametrize("shape,lattice", [((6, 5, 128), "D3Q19"), ((4, 3, 256), "D3Q19"),
                                           ((5, 4, 160), "D3Q19"), ((40, 256), "D2Q9")])
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f64"])
@pytest.mark.parametrize("kind", ["force", "faces", "pressure"])
def test_staged_equals_global_gather(shape, lattice, storage, kind):
    from maddening_b200.batched import LBMEnsemble
    node, st, bi = _node(shape, storage, lattice, kind)
    staged = node.run(st, bi, 9)
    plain = LBMEnsemble([node]).run([st], [bi], 9)[0]
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.equal(staged[key], plain[key]), key


def test_staged_matches_oracle_fp64():
    node, st, bi = _node((5, 4, 160), "f64", "D3Q19", "pressure")
    out = node.run(st, bi, 6)
    orc = R.OracleLBM((5, 4, 160), 0.05, "D3Q19", wall_mask=node._wall_np)
    so = orc.initial_state()
    so["f"] = st["f"].cpu().numpy()
    so = orc.run(so, bi, 6)
    np.testing.assert_allclose(out["f"].cpu().numpy(), so["f"], rtol=0, atol=1e-14)


def test_staged_status_word_stays_clear():
    from maddening_b200 import _lib
    node, st, bi = _node((8, 8, 256), "f32", "D3Q19", "force")
    plan = node.plan
    args, keep = node._step_args(st, bi, torch.device("cuda"))
    f_out, rho, vel, prs, mom = node._outputs(torch.device("cuda"))
    ws = torch.zeros(plan.workspace_bytes(), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().lbm_rollout(plan.handle, stream, st["f"].data_ptr(), f_out.data_ptr(),
                                      20, C.byref(args), C.byref(mom), ws.data_ptr(), ws.numel()))
    torch.cuda.synchronize()
    sb = (plan.state_bytes() + 255) // 256 * 256
    status = int(ws[2 * sb: 2 * sb + 4].view(torch.int32).item())
    assert status == 0
