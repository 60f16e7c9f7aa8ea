"""The reference's LBM tests, run on the B200 node with the same assertions.

Sources: tests/nodes/test_lbm.py (finite step 195-215, equilibrium stability
222-241, 2-D Poiseuille with Zou-He faces 248-329, periodic mass 336-357,
wall velocity 364-387, clot injection 419-453, fluxes 515-520) and
tests/cloud/multigpu/test_lbm_poiseuille.py (pipe Poiseuille amplitude,
70-162, run unsharded).
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _node(**kw):
    from maddening_b200 import LBMNode
    return LBMNode(**kw)


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("grid,lattice", [((8, 8, 8), "D3Q19"), ((16, 8), "D2Q9")])
def test_step_produces_finite(grid, lattice):
    node = _node(name="lbm", timestep=0.001, grid_shape=grid, lattice=lattice)
    st = node.update(node.initial_state(), {}, node.delta_t)
    for key in ("f", "density", "velocity", "pressure"):
        assert torch.isfinite(st[key]).all(), key


def test_initial_state_matches_reference_contract():
    node = _node(name="lbm", timestep=0.001, grid_shape=(8, 6, 4))
    st = node.initial_state()
    assert tuple(st["f"].shape) == (8, 6, 4, 19) and st["f"].dtype == torch.float32
    assert tuple(st["velocity"].shape) == (8, 6, 4, 3)
    assert st["wall_mask"].dtype == torch.uint8
    np.testing.assert_allclose(_np(st["density"]), 1.0, rtol=1e-5)
    np.testing.assert_allclose(_np(st["pressure"]), 1.0 / 3.0, rtol=1e-5)
    np.testing.assert_allclose(_np(st["f"].sum(-1)), _np(st["density"]), rtol=1e-5)
    np.testing.assert_array_equal(_np(st["f"][0, 0, 0]), node.lattice.w.astype(np.float32))


@pytest.mark.parametrize("grid,lattice", [((8, 8, 8), "D3Q19"), ((16, 16), "D2Q9")])
@pytest.mark.parametrize("fused", [False, True])
def test_equilibrium_stays_stable(grid, lattice, fused):
    node = _node(name="lbm", timestep=0.001, grid_shape=grid, lattice=lattice)
    st = node.initial_state()
    if fused:
        st = node.run(st, {}, 100)
    else:
        for _ in range(100):
            st = node.update(st, {}, node.delta_t)
    np.testing.assert_allclose(_np(st["density"]), 1.0, rtol=1e-3)
    np.testing.assert_allclose(_np(st["velocity"]), 0.0, atol=1e-4)


@pytest.mark.parametrize("fused", [False, True])
def test_poiseuille_2d_zou_he(fused):
    nx, ny = 64, 16
    wall = np.zeros((nx, ny), dtype=bool)
    wall[:, 0] = True
    wall[:, ny - 1] = True
    viscosity = 0.1
    node = _node(name="poiseuille", timestep=0.001, grid_shape=(nx, ny), viscosity=viscosity,
                 lattice="D2Q9", wall_mask=wall, inlet_face="x_min", outlet_face="x_max")
    st = node.initial_state()
    bi = {"inlet_pressure": np.float32(1.0 / 3.0 * 1.01),
          "outlet_pressure": np.float32(1.0 / 3.0 * 1.00)}
    if fused:
        st = node.run(st, bi, 2000)
    else:
        for _ in range(2000):
            st = node.update(st, bi, node.delta_t)
    assert torch.isfinite(st["velocity"]).all()
    u = _np(st["velocity"][nx // 2, :, 0])
    np.testing.assert_allclose(u[0], 0.0, atol=1e-6)
    np.testing.assert_allclose(u[ny - 1], 0.0, atol=1e-6)
    ui = u[1:ny - 1]
    assert np.all(ui > 0)
    assert abs(int(np.argmax(ui)) + 1 - ny // 2) <= 2
    H = ny - 2
    dp_dx = (1.01 - 1.0) / nx
    y = np.arange(1, ny - 1) - 0.5
    ua = dp_dx / (2.0 * viscosity) * y * (H - y)
    np.testing.assert_allclose(ui / ui.max(), ua / ua.max(), atol=0.15)


@pytest.mark.parametrize("fused", [False, True])
def test_mass_conserved_periodic(fused):
    node = _node(name="lbm", timestep=0.001, grid_shape=(16, 16, 16), viscosity=0.1)
    st = node.initial_state()
    m0 = float(st["density"].double().sum())
    if fused:
        st = node.run(st, {}, 50)
    else:
        for _ in range(50):
            st = node.update(st, {}, node.delta_t)
    np.testing.assert_allclose(float(st["density"].double().sum()), m0, rtol=1e-5)
    mm = _np(node.mass_momentum(st["f"]))
    np.testing.assert_allclose(mm[0], 16 ** 3, rtol=1e-6)


def test_wall_cells_have_zero_velocity():
    wall = np.zeros((8, 8, 8), dtype=bool)
    wall[3:5] = True
    node = _node(name="lbm", timestep=0.001, grid_shape=(8, 8, 8), wall_mask=wall)
    st = node.initial_state()
    force = torch.zeros((8, 8, 8, 3), device="cuda")
    force[..., 0] = 0.001
    for _ in range(20):
        st = node.update(st, {"body_force": force}, node.delta_t)
    np.testing.assert_allclose(_np(st["velocity"][3:5]), 0.0, atol=1e-10)


def test_clot_injection_wall_mask_update():
    node = _node(name="lbm", timestep=0.001, grid_shape=(16, 8, 8), viscosity=0.1)
    st = node.initial_state()
    force = torch.zeros((16, 8, 8, 3), device="cuda")
    force[..., 0] = 0.0005
    for _ in range(10):
        st = node.update(st, {"body_force": force}, node.delta_t)
    assert float(st["velocity"][8, 3:5, 3:5, 0].abs().mean()) > 1e-6
    clot = np.zeros((16, 8, 8), dtype=bool)
    clot[8, 3:5, 3:5] = True
    for _ in range(10):
        st = node.update(st, {"body_force": force, "wall_mask_update": clot}, node.delta_t)
    np.testing.assert_allclose(_np(st["velocity"][8, 3:5, 3:5, :]), 0.0, atol=1e-10)


def test_compute_boundary_fluxes():
    node = _node(name="lbm", timestep=0.001, grid_shape=(8, 8, 8))
    st = node.initial_state()
    fl = node.compute_boundary_fluxes(st, {}, node.delta_t)
    assert torch.isfinite(fl["outlet_pressure_avg"])
    np.testing.assert_allclose(float(fl["outlet_pressure_avg"]), 1.0 / 3.0, rtol=1e-6)


def _cylinder_mask(nx, ny, nz, radius):
    yy = np.arange(ny) - (ny - 1) / 2.0
    zz = np.arange(nz) - (nz - 1) / 2.0
    Y, Z = np.meshgrid(yy, zz, indexing="ij")
    return np.broadcast_to((Y * Y + Z * Z > radius * radius)[None], (nx, ny, nz)).copy()


def test_pipe_poiseuille_amplitude():
    """Centre-line velocity / (F R^2 / 4 mu) within (0.75, 1.30) after 500 steps."""
    nx, ny, nz, R, nu, F = 4, 12, 12, 4.0, 0.1, 1e-4
    node = _node(name="pois", timestep=1.0, grid_shape=(nx, ny, nz), viscosity=nu,
                 wall_mask=_cylinder_mask(nx, ny, nz, R))
    st = node.run(node.initial_state(),
                  {"body_force": np.array([F, 0.0, 0.0], dtype=np.float32)}, 500)
    ux = _np(st["velocity"][..., 0]).mean(axis=0)
    cy, cz = (ny - 1) // 2, (nz - 1) // 2
    yy = np.arange(ny) - (ny - 1) / 2.0
    Y, Z = np.meshgrid(yy, yy, indexing="ij")
    r = np.sqrt(Y * Y + Z * Z)
    fluid = r <= R - 0.5
    assert ux[fluid].min() > 0
    np.testing.assert_allclose(ux[cy, cz], ux[fluid].max(), rtol=1e-5)
    ratio = ux[cy, cz] / (F * R * R / (4.0 * nu))
    assert 0.75 < ratio < 1.30, ratio
    np.testing.assert_allclose(ux[cy, cz], ux[cy + 1, cz], rtol=1e-3)
