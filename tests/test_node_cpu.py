"""Host-side behaviour of the node (no GPU): construction, validation, contract.

Mirrors tests/nodes/test_lbm.py:103-142 (construction) and 499-520 (spec).
"""

import numpy as np
import pytest

from maddening_b200 import LBMNode, d2q9, d3q19


def test_default_3d():
    node = LBMNode(name="lbm", timestep=0.001, grid_shape=(8, 8, 8))
    assert node.name == "lbm" and node._D == 3 and node._Q == 19 and node.tau > 0.5


def test_2d():
    node = LBMNode(name="lbm2d", timestep=0.001, grid_shape=(16, 8), lattice="D2Q9")
    assert node._D == 2 and node._Q == 9


def test_invalid_lattice():
    with pytest.raises(ValueError, match="Unknown lattice"):
        LBMNode(name="x", timestep=0.001, grid_shape=(8, 8, 8), lattice="D1Q3")


def test_grid_shape_mismatch():
    with pytest.raises(ValueError, match="dims"):
        LBMNode(name="x", timestep=0.001, grid_shape=(8, 8), lattice="D3Q19")


def test_viscosity_sets_tau():
    node = LBMNode(name="lbm", timestep=0.001, grid_shape=(8, 8, 8), viscosity=0.15)
    np.testing.assert_allclose(node.tau, 0.5 + 0.15 / (1.0 / 3.0), rtol=1e-10)
    np.testing.assert_allclose(node.viscosity, 0.15, rtol=1e-12)


def test_tau_must_exceed_half():
    with pytest.raises(ValueError, match="tau must be > 0.5"):
        LBMNode(name="x", timestep=0.001, grid_shape=(8, 8, 8), viscosity=0.0)


def test_wall_mask_shape_validation():
    with pytest.raises(ValueError, match="wall_mask shape"):
        LBMNode(name="x", timestep=0.001, grid_shape=(8, 8, 8),
                wall_mask=np.zeros((4, 4, 4), dtype=bool))


@pytest.mark.parametrize("face", ["z_min", "w_max"])
def test_face_validation(face):
    with pytest.raises(ValueError):
        LBMNode(name="x", timestep=0.001, grid_shape=(8, 8), lattice="D2Q9", inlet_face=face)


def test_halo_and_spec():
    node = LBMNode(name="lbm", timestep=0.001, grid_shape=(8, 8, 8))
    assert node.halo_width() == {0: 1, 1: 1, 2: 1}
    assert node.requires_halo is True
    n2 = LBMNode(name="lbm", timestep=0.001, grid_shape=(8, 8), lattice="D2Q9")
    assert n2.halo_width() == {0: 1, 1: 1}
    spec = node.boundary_input_spec()
    for k in ("inlet_pressure", "outlet_pressure", "body_force", "wall_mask_update"):
        assert k in spec
    assert spec["body_force"].coupling_type == "additive"
    assert spec["body_force"].shape == (8, 8, 8, 3)


def test_derivatives_raises():
    node = LBMNode(name="lbm", timestep=0.001, grid_shape=(8, 8, 8))
    with pytest.raises(NotImplementedError, match="discrete"):
        node.derivatives({}, {})


def test_update_padded_needs_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    node = LBMNode(name="lbm", timestep=0.001, grid_shape=(8, 8, 8))
    with pytest.raises(RuntimeError, match="CUDA"):
        node.update_padded({"f": np.zeros((10, 10, 10, 19), np.float32)}, {}, 1.0)


def test_lattice_descriptors_match_reference_order():
    lat = d3q19()
    assert lat.Q == 19 and lat.D == 3 and lat.e.shape == (19, 3)
    np.testing.assert_allclose(lat.w.sum(), 1.0, rtol=1e-12)
    for q in range(lat.Q):
        assert lat.opp[lat.opp[q]] == q
        np.testing.assert_array_equal(lat.e[lat.opp[q]], -lat.e[q])
    lat2 = d2q9()
    np.testing.assert_allclose(lat2.w[0], 4.0 / 9.0)
    assert isinstance(lat.e, np.ndarray)


def test_no_cpu_path():
    import torch
    if torch.cuda.is_available():
        pytest.skip("has a GPU")
    node = LBMNode(name="lbm", timestep=0.001, grid_shape=(8, 8, 8))
    with pytest.raises(RuntimeError, match="CUDA"):
        node.initial_state()


def test_one_pass_choice_sets_plan_flags():
    """``one_pass`` None / True keep the library's one pass; False asks for two."""
    from maddening_b200 import LBMNode, _lib
    for storage in ("f32", "f16", "bf16"):
        for one in (None, True):
            node = LBMNode("n", 1.0, grid_shape=(8, 8, 8), storage=storage, one_pass=one)
            assert node.plan.flags & _lib.PLAN_TWO_PASS == 0
        assert LBMNode("n", 1.0, grid_shape=(8, 8, 8), storage=storage,
                       one_pass=False).plan.flags & _lib.PLAN_TWO_PASS
