"""Paired-cell state step (two neighbouring cells per thread, 32/64-bit plane
accesses, shuffles for the pull along the contiguous axis): bit-identical to
the one-cell step for every storage form, lattice, face axis and force mode,
including the periodic wrap at both ends of a row and every warp/block width
(contiguous extents 64, 128, 192, 256); the instance-wide pair form for other
even rows (rows shorter than a warp, pairs whose neighbour lies in the next
row, a partial last warp); the four-cell form of 16-bit storage (rows of
128, 256, 384, 512 cells; D2Q9 rows of any multiple of 4); odd rows fall back to
the one-cell step."""

import numpy as np
import pytest
import torch

from oracle import lbm_ref as R

pytestmark = pytest.mark.gpu


def _node(shape, storage, lattice, kind, cpt, seed=0):
    from maddening_b200 import LBMNode
    rng = np.random.default_rng(seed)
    wall = rng.random(shape) < 0.08
    kw, bi = {}, {}
    D = len(shape)
    if kind == "faces":
        wall[0] = wall[-1] = False
        kw = dict(outlet_condition="zero_gradient")
        bi = {"inlet_velocity": np.array([0.04] + [0.0] * (D - 1))}
    elif kind == "faces_contiguous":
        # faces on the last (contiguous) axis: the row ends of every warp segment
        wall[..., 0] = wall[..., -1] = False
        face = "z" if D == 3 else "y"
        kw = dict(outlet_condition="zero_gradient", inlet_face=f"{face}_min",
                  outlet_face=f"{face}_max")
        bi = {"inlet_velocity": np.array([0.0] * (D - 1) + [0.03]),
              "body_force": np.array([1e-5] + [0.0] * (D - 1), dtype=np.float32)}
    elif kind == "pressure":
        wall[0] = wall[-1] = False
        bi = {"inlet_pressure": np.float32(1 / 3 + 1e-3), "outlet_pressure": np.float32(1 / 3),
              "body_force": rng.uniform(-1e-5, 1e-5, shape + (D,)).astype(np.float32)}
    else:
        bi = {"body_force": np.array([1e-5, -2e-6, 3e-6][:D], dtype=np.float32)}
    node = LBMNode("p", 1.0, grid_shape=shape, viscosity=0.05, lattice=lattice, wall_mask=wall,
                   storage=storage, cells_per_thread=cpt, **kw)
    st = node.initial_state()
    lat = node.lattice
    st["f"] = torch.as_tensor(lat.w * (1 + 1e-3 * rng.standard_normal(shape + (lat.Q,))),
                              device="cuda").to(st["f"].dtype)
    return node, st, bi


@pytest.mark.parametrize("shape,lattice", [((6, 5, 64), "D3Q19"), ((4, 3, 256), "D3Q19"),
                                           ((3, 4, 128), "D3Q19"), ((5, 2, 192), "D3Q19"),
                                           ((1, 1, 64), "D3Q19"), ((40, 128), "D2Q9"),
                                           ((24, 256), "D2Q9"), ((9, 512), "D2Q9"),
                                           ((7, 384), "D2Q9"),
                                           # instance-wide four-cell form (D2Q9)
                                           ((31, 36), "D2Q9"), ((5, 100), "D2Q9"),
                                           ((3, 4), "D2Q9"),
                                           # instance-wide pairs (even rows)
                                           ((3, 4, 100), "D3Q19"), ((5, 3, 34), "D3Q19"),
                                           ((4, 7, 2), "D3Q19"), ((33, 38), "D2Q9"),
                                           # odd rows: one-cell fallback
                                           ((5, 6, 37), "D3Q19"), ((33, 19), "D2Q9")])
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("kind", ["force", "faces", "faces_contiguous", "pressure"])
def test_paired_equals_single(shape, lattice, storage, kind):
    if shape[0] == 1 and kind in ("faces", "pressure"):
        pytest.skip("x faces need more than one cell along x")
    if shape[-1] < 3 and kind == "faces_contiguous":
        pytest.skip("a zero-gradient face needs three cells along its axis")
    node2, st, bi = _node(shape, storage, lattice, kind, 2)
    node1, _, _ = _node(shape, storage, lattice, kind, 1)
    a = node2.run(st, bi, 7)
    b = node1.run(st, bi, 7)
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.equal(a[key], b[key]), key


def test_paired_default_for_16bit_matches_single():
    node0, st, bi = _node((4, 6, 128), "f16", "D3Q19", "faces", None)
    node1, _, _ = _node((4, 6, 128), "f16", "D3Q19", "faces", 1)
    a = node0.run(st, bi, 5)
    b = node1.run(st, bi, 5)
    assert torch.equal(a["f"], b["f"])


def test_paired_fp32_matches_oracle():
    shape = (5, 4, 64)
    node, st, bi = _node(shape, "f32", "D3Q19", "pressure", 2)
    out = node.run(st, bi, 6)
    orc = R.OracleLBM(shape, 0.05, "D3Q19", wall_mask=node._wall_np)
    so = orc.initial_state()
    so["f"] = st["f"].cpu().numpy().astype(np.float64)
    so = orc.run(so, bi, 6)
    np.testing.assert_allclose(out["f"].cpu().numpy(), so["f"], rtol=0, atol=1e-6)
    assert R.rel_l2(out["velocity"].cpu().numpy(), so["velocity"]) < 1e-5
