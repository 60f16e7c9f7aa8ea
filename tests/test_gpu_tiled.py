"""One-pass tiled step (``k_tiled``): ``update`` reads the reference-layout
``f`` once, collides each plane of a column in shared memory and pulls from
it; the first step of ``run`` does the same and writes the next state.

Both must equal the two-pass path (collide into the workspace, then the pull
step) bit for bit: every lattice form, storage, force mode and face
condition, on lattices with partial tiles, wrap-around halos and extents of
one to three cells.  Its bounded waits are made to run out through the test
hook ``LBM_PLAN_TEST_WAIT_TIMEOUT`` (barriers armed, no copies issued): the
kernel sets the status word and returns, and the context stays usable.
"""

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SHAPES_3D = [(16, 8, 32), (20, 10, 36), (12, 10, 16), (7, 9, 68), (5, 17, 100), (3, 1, 4),
             (1, 3, 8)]
SHAPES_2D = [(16, 32), (37, 260), (100, 1028), (3, 4)]
KINDS = ["uniform", "field", "inlet_zero_gradient", "pressure_last_axis",
         "zero_gradient_mid_axis"]


def _case(shape, lattice, storage, kind, one_pass, seed=0):
    from maddening_b200 import LBMNode
    rng = np.random.default_rng(seed)
    D = len(shape)
    wall = rng.random(shape) < 0.1
    kw, bi = {}, {}
    if kind == "uniform":
        bi = {"body_force": np.array([1e-5, -2e-6, 3e-6][:D], dtype=np.float32)}
    elif kind == "field":
        bi = {"body_force": rng.uniform(-1e-5, 1e-5, shape + (D,)).astype(np.float32)}
    elif kind == "inlet_zero_gradient":  # the benchmark's faces, on axis 0
        kw = dict(inlet_face="x_min", outlet_face="x_max", outlet_condition="zero_gradient")
        bi = {"inlet_velocity": np.array([0.05] + [0.0] * (D - 1), dtype=np.float32)}
    elif kind == "pressure_last_axis":
        last = "z" if D == 3 else "y"
        kw = dict(inlet_face=f"{last}_min", outlet_face=f"{last}_max")
        bi = {"inlet_pressure": np.float32(1 / 3 + 2e-3), "outlet_pressure": np.float32(1 / 3),
              "body_force": np.array([2e-6, 1e-6, 0.0][:D], dtype=np.float32)}
    elif kind == "zero_gradient_mid_axis":
        mid = "y" if D == 3 else "x"
        kw = dict(inlet_face=f"{mid}_max", outlet_face=f"{mid}_min",
                  outlet_condition="zero_gradient")
        u = [0.0, -0.03, 0.01] if D == 3 else [-0.03, 0.01]
        bi = {"inlet_velocity": np.array(u, dtype=np.float32),
              "body_force": rng.uniform(-1e-5, 1e-5, shape + (D,)).astype(np.float32)}
    node = LBMNode("t", 1.0, grid_shape=shape, viscosity=0.06, lattice=lattice, wall_mask=wall,
                   storage=storage, one_pass=one_pass, **kw)
    st = node.initial_state()
    lat = node.lattice
    st["f"] = torch.as_tensor(lat.w * (1 + 1e-3 * rng.standard_normal(shape + (lat.Q,))),
                              device="cuda").to(st["f"].dtype)
    return node, st, bi


def _face_axis_long_enough(kind, shape):
    if kind == "inlet_zero_gradient":
        return shape[0] >= 3
    if kind == "pressure_last_axis":
        return shape[-1] >= 2
    if kind == "zero_gradient_mid_axis":
        return shape[1 if len(shape) == 3 else 0] >= 3
    return True


@pytest.mark.parametrize("shape,lattice", [(s, "D3Q19") for s in SHAPES_3D] +
                         [(s, "D2Q9") for s in SHAPES_2D])
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("kind", KINDS)
def test_one_pass_update_equals_two_pass(shape, lattice, storage, kind):
    if not _face_axis_long_enough(kind, shape):
        pytest.skip("face axis too short for this condition")
    a, st, bi = _case(shape, lattice, storage, kind, True)
    b, _, _ = _case(shape, lattice, storage, kind, False)
    x = a.update(st, bi, 1.0)
    y = b.update(st, bi, 1.0)
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.equal(x[key], y[key]), key


@pytest.mark.parametrize("shape,lattice", [((20, 10, 36), "D3Q19"), ((7, 9, 68), "D3Q19"),
                                           ((37, 260), "D2Q9")])
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("kind", ["field", "inlet_zero_gradient"])
def test_one_pass_first_step_of_run_equals_two_pass(shape, lattice, storage, kind):
    a, st, bi = _case(shape, lattice, storage, kind, True, seed=3)
    b, _, _ = _case(shape, lattice, storage, kind, False, seed=3)
    for n in (2, 7):
        x = a.run(st, bi, n)
        y = b.run(st, bi, n)
        for key in ("f", "density", "velocity", "pressure"):
            assert torch.equal(x[key], y[key]), (n, key)


def test_one_pass_update_at_256_cube_equals_two_pass():
    """The benchmark's lattice: 256 columns swept in chunks by 148 blocks."""
    from maddening_b200 import LBMNode
    from maddening_b200.geometry import random_spheres
    shape = (256, 256, 256)
    kw = dict(grid_shape=shape, viscosity=0.1 / 3, wall_mask=random_spheres(shape, seed=0),
              outlet_condition="zero_gradient")
    a = LBMNode("a", 1.0, **kw)
    b = LBMNode("b", 1.0, one_pass=False, **kw)
    bi = {"inlet_velocity": np.array([0.05, 0.0, 0.0], dtype=np.float32)}
    st = a.run(a.initial_state(), bi, 3)
    x = a.update(st, bi, 1.0)
    y = b.update(st, bi, 1.0)
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.equal(x[key], y[key]), key


def test_in_place_update_takes_two_passes():
    """f_out == f_in cannot be swept in one pass (other blocks still read f_in):
    the call falls back to the two-pass path and gives the same result."""
    from maddening_b200 import _lib
    node, st, bi = _case((12, 10, 16), "D3Q19", "f32", "field", True, seed=2)
    ref = node.update(st, bi, 1.0)
    dev = torch.device("cuda")
    args, keep = node._step_args(st, bi, dev)
    _f, rho, vel, prs, mom = node._outputs(dev)
    f = st["f"].clone()
    ws = torch.empty(node.plan.state_bytes(), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().lbm_update(node.plan.handle, stream, f.data_ptr(), f.data_ptr(),
                                     C.byref(args), C.byref(mom), ws.data_ptr(), ws.numel()))
    torch.cuda.synchronize()
    assert torch.equal(f, ref["f"]) and torch.equal(rho, ref["density"])


def test_wait_timeout_sets_status_and_returns():
    """Barriers armed, no copy issued: the waits give up after their time
    limit, the kernel records it in the status word (the first 4 bytes of an
    update's workspace) and returns; the next call on the same stream runs
    normally."""
    from maddening_b200 import _lib
    shape = (20, 10, 36)
    node, st, bi = _case(shape, "D3Q19", "f32", "inlet_zero_gradient", True, seed=4)
    hook = _lib.Plan(19, shape, node.tau, "f32", flags=_lib.PLAN_TEST_WAIT_TIMEOUT)
    dev = torch.device("cuda")
    args, keep = node._step_args(st, bi, dev)
    _f, rho, vel, prs, mom = node._outputs(dev)
    f_in = st["f"].contiguous()
    f_out = torch.zeros_like(f_in)
    ws = torch.full((node.plan.state_bytes(),), 0x55, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().lbm_update(hook.handle, stream, f_in.data_ptr(), f_out.data_ptr(),
                                     C.byref(args), C.byref(mom), ws.data_ptr(), ws.numel()))
    torch.cuda.synchronize()
    assert int(ws[:4].view(torch.int32).item()) == 1
    # the same stream, normal plans: the context is intact
    ref = node.update(st, bi, 1.0)
    two = _case(shape, "D3Q19", "f32", "inlet_zero_gradient", False, seed=4)[0]
    assert torch.equal(ref["f"], two.update(st, bi, 1.0)["f"])


def test_status_word_clear_after_normal_update():
    from maddening_b200 import _lib
    node, st, bi = _case((16, 8, 32), "D3Q19", "f32", "uniform", True)
    dev = torch.device("cuda")
    args, keep = node._step_args(st, bi, dev)
    f_out, rho, vel, prs, mom = node._outputs(dev)
    ws = torch.full((node.plan.state_bytes(),), 0x55, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().lbm_update(node.plan.handle, stream, st["f"].data_ptr(),
                                     f_out.data_ptr(), C.byref(args), C.byref(mom),
                                     ws.data_ptr(), ws.numel()))
    torch.cuda.synchronize()
    assert int(ws[:4].view(torch.int32).item()) == 0
