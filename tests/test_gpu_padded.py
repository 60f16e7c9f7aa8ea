"""Halo-padded step ``LBMNode.update_padded`` (the reference's lbm.py:747-897)
through ``lbm_update_padded``.

* golden cases: the reference's own ``update_padded`` executed on padded
  states whose halos are a periodic pad or foreign data (standing in for a
  neighbour shard); FP32 within float32 rounding of the x64 run, FP64 storage
  within 1e-12;
* the reference's own check (``tests/nodes/test_lbm_stream_padded.py:66-186``):
  with a periodic pad on every axis the interior equals ``update`` -- here bit
  for bit, the kernels share their arithmetic -- for walls, force fields,
  pressure faces and the face extensions;
* halo entries of every output keep the input's values.
"""

import numpy as np
import pytest
import torch

from tests.golden.make_golden import PADDED_CASES

pytestmark = pytest.mark.gpu

F32_EPS = float(np.finfo(np.float32).eps)


def _node_for(case, storage="f32", **kw):
    from maddening_b200 import LBMNode
    return LBMNode(case["name"], 1.0, grid_shape=case["grid"], viscosity=case["viscosity"],
                   lattice=case["lattice"], inlet_face=case["faces"][0],
                   outlet_face=case["faces"][1], storage=storage, **kw)


def _padded_state(golden, case, storage):
    p = f"{case['name']}|x64|"
    dt = torch.float64 if storage == "f64" else torch.float32
    st = {"f": torch.as_tensor(golden[p + "f_pad"].astype(np.float64), device="cuda").to(dt),
          "density": torch.as_tensor(golden[p + "density_pad"], device="cuda"),
          "velocity": torch.as_tensor(golden[p + "velocity_pad"], device="cuda"),
          "pressure": torch.as_tensor(golden[p + "pressure_pad"], device="cuda"),
          "wall_mask": torch.as_tensor(golden[p + "wall_pad"], device="cuda")}
    bi = {}
    for k in golden.files:
        if k.startswith(p + "bi_"):
            v = golden[k]
            bi[k[len(p) + 3:]] = np.float32(v) if v.ndim == 0 else v
    return st, bi, p


def _np(t):
    return t.detach().cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("case", PADDED_CASES, ids=[c["name"] for c in PADDED_CASES])
def test_update_padded_matches_reference(golden, case):
    node = _node_for(case)
    st, bi, p = _padded_state(golden, case, "f32")
    out = node.update_padded(st, bi, 1.0)
    ref_f = golden[p + "out_f"]
    assert np.max(np.abs(_np(out["f"]) - ref_f) / np.abs(ref_f)) <= 4 * F32_EPS
    for key, tol in (("density", 4e-7), ("velocity", 4e-7), ("pressure", 2e-7)):
        err = np.max(np.abs(_np(out[key]) - golden[p + "out_" + key]))
        assert err <= tol, (key, err)


@pytest.mark.parametrize("case", PADDED_CASES, ids=[c["name"] for c in PADDED_CASES])
def test_update_padded_fp64_storage_matches_reference(golden, case):
    node = _node_for(case, storage="f64")
    st, bi, p = _padded_state(golden, case, "f64")
    out = node.update_padded(st, bi, 1.0)
    for key in ("f", "density", "velocity", "pressure"):
        err = np.max(np.abs(_np(out[key]) - golden[p + "out_" + key]))
        # density/velocity/pressure keep the input's float32 halo entries
        assert err <= 1e-12 if key == "f" else err <= 1e-7, (key, err)


def _pad(t, extra=0):
    """Periodic pad by one cell on every spatial axis (a single-device halo)."""
    D = t.ndim - extra
    for d in range(D):
        t = torch.cat([t.narrow(d, t.shape[d] - 1, 1), t, t.narrow(d, 0, 1)], dim=d)
    return t.contiguous()


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("kind", ["walls_force_field", "pressure", "velocity_zero_gradient",
                                  "d2q9"])
def test_periodic_pad_interior_equals_update(storage, kind):
    from maddening_b200 import LBMNode
    rng = np.random.default_rng(11)
    lattice, grid = ("D2Q9", (9, 12)) if kind == "d2q9" else ("D3Q19", (7, 6, 9))
    D = len(grid)
    wall = rng.random(grid) < 0.12
    kw, bi = {}, {}
    if kind in ("pressure", "velocity_zero_gradient", "d2q9"):
        wall[0] = wall[-1] = False
    if kind in ("walls_force_field", "d2q9"):
        bi["body_force"] = (1e-5 * rng.standard_normal(grid + (D,))).astype(np.float32)
    if kind in ("pressure", "d2q9"):
        bi["inlet_pressure"] = np.float32(1 / 3 + 1e-3)
        bi["outlet_pressure"] = np.float32(1 / 3)
    if kind == "velocity_zero_gradient":
        kw = dict(outlet_condition="zero_gradient")
        bi["inlet_velocity"] = np.array([0.03] + [0.0] * (D - 1))
    node = LBMNode("pad", 1.0, grid_shape=grid, viscosity=0.07, lattice=lattice,
                   wall_mask=wall, storage=storage, **kw)
    st = node.initial_state()
    lat = node.lattice
    f0 = lat.w * (1 + 1e-3 * rng.standard_normal(grid + (lat.Q,)))
    st["f"] = torch.as_tensor(f0, device="cuda").to(st["f"].dtype)
    ref = node.update(st, bi, 1.0)
    stp = {"f": _pad(st["f"], 1), "density": _pad(st["density"]),
           "velocity": _pad(st["velocity"], 1), "pressure": _pad(st["pressure"]),
           "wall_mask": _pad(st["wall_mask"])}
    bip = dict(bi)
    if "body_force" in bi:   # padded periodically: the halo cells collide with their force
        bip["body_force"] = _pad(torch.as_tensor(bi["body_force"], device="cuda"), 1)
    out = node.update_padded(stp, bip, 1.0)
    inner = (slice(1, -1),) * D
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.equal(out[key][inner], ref[key]), key
    # halo entries: the input's
    halo = torch.ones(stp["density"].shape, dtype=torch.bool, device="cuda")
    halo[inner] = False
    assert torch.equal(out["f"][halo], stp["f"][halo])
    assert torch.equal(out["density"][halo], stp["density"][halo])
    assert torch.equal(out["velocity"][halo], stp["velocity"][halo])


def test_interior_force_field_is_zero_padded():
    """An interior-shaped body force is zero-padded (lbm.py:826-832): the same
    result as passing the zero-padded field explicitly."""
    from maddening_b200 import LBMNode
    rng = np.random.default_rng(5)
    grid = (6, 5, 7)
    node = LBMNode("pad", 1.0, grid_shape=grid, viscosity=0.1)
    st = node.initial_state()
    st["f"] = torch.as_tensor(node.lattice.w * (1 + 1e-3 * rng.standard_normal(grid + (19,))),
                              device="cuda").float()
    stp = {"f": _pad(st["f"], 1), "density": _pad(st["density"]),
           "velocity": _pad(st["velocity"], 1), "pressure": _pad(st["pressure"]),
           "wall_mask": _pad(st["wall_mask"])}
    F = torch.as_tensor(1e-5 * rng.standard_normal(grid + (3,)), device="cuda").float()
    Fz = torch.zeros((8, 7, 9, 3), device="cuda")
    Fz[1:-1, 1:-1, 1:-1] = F
    a = node.update_padded(stp, {"body_force": F}, 1.0)
    b = node.update_padded(stp, {"body_force": Fz}, 1.0)
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.equal(a[key], b[key]), key
