"""Reference-layout inputs and outputs (*grid, Q) move block by block through
shared memory, with 16-byte loads and stores when the array is 16-byte
aligned and plain coalesced ones otherwise.  Both give the same bytes: a
rollout read from and written to arrays shifted by one element (so never
16-byte aligned) equals the aligned one, on lattices whose cell count leaves
a partial last block."""

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,lattice", [((5, 7, 9), "D3Q19"), ((3, 3, 136), "D3Q19"),
                                           ((13, 11), "D2Q9")])
@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
def test_unaligned_output_equals_aligned(shape, lattice, storage):
    from maddening_b200 import LBMNode, _lib
    rng = np.random.default_rng(5)
    wall = rng.random(shape) < 0.1
    node = LBMNode("a", 1.0, grid_shape=shape, viscosity=0.07, lattice=lattice, wall_mask=wall,
                   storage=storage)
    st = node.initial_state()
    lat = node.lattice
    st["f"] = torch.as_tensor(lat.w * (1 + 1e-3 * rng.standard_normal(shape + (lat.Q,))),
                              device="cuda").to(st["f"].dtype)
    D = len(shape)
    bi = {"body_force": np.array([1e-5, -3e-6, 2e-6][:D], dtype=np.float32)}
    ref = node.run(st, bi, 5)
    dev = torch.device("cuda")
    args, keep = node._step_args(st, bi, dev)
    _f, rho, vel, prs, mom = node._outputs(dev)
    n = st["f"].numel()
    big = torch.full((n + 1,), float("nan"), dtype=st["f"].dtype, device=dev)
    f_out = big[1:]  # one element past a 256-byte boundary
    assert f_out.data_ptr() % 16 != 0
    big_in = torch.empty((n + 1,), dtype=st["f"].dtype, device=dev)
    f_in = big_in[1:]
    f_in.copy_(st["f"].reshape(-1))
    assert f_in.data_ptr() % 16 != 0
    ws = torch.empty(node.plan.workspace_bytes(), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().lbm_rollout(node.plan.handle, stream, f_in.data_ptr(),
                                      f_out.data_ptr(), 5, C.byref(args), C.byref(mom),
                                      ws.data_ptr(), ws.numel()))
    torch.cuda.synchronize()
    assert torch.equal(f_out.view(ref["f"].shape), ref["f"])
    assert torch.equal(rho, ref["density"]) and torch.equal(vel, ref["velocity"])
    assert torch.isnan(big[0])  # nothing written before the output
