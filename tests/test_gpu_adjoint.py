"""The hand-written adjoint of the rollout (``LBMNode.rollout`` backward).

Checked against
* autograd of the torch restatement of the reference step (standing in for
  ``jax.grad`` of the reference node): FP64 adjoint to 1e-9, FP32 to 1e-4;
* central finite differences of the FP64 forward;
* the differentiated-rollout configuration: 128^3 D3Q19, z walls, tau 0.7,
  force field 1e-6 N(0,1), loss = final kinetic energy after 1000 steps,
  checkpoint every 32 steps: FP32 adjoint vs central differences of the FP64
  forward (eps = 1e-3 relative to max(|F|, 1e-6)) on 16 random cells,
  relative error <= 1e-4.
"""

import numpy as np
import pytest
import torch

from oracle import lbm_ref as R
from oracle import lbm_ref_torch as RT

pytestmark = pytest.mark.gpu


def _kinetic(out):
    return 0.5 * (out["density"] * (out["velocity"] ** 2).sum(-1)).sum()


def _case(lattice, grid, seed, force_kind):
    rng = np.random.default_rng(seed)
    lat = R.lattice(lattice)
    D = lat.D
    wall = rng.random(grid) < 0.15
    wall[..., 0] = True
    f0 = lat.w * (1.0 + 2e-3 * rng.standard_normal(grid + (lat.Q,)))
    if force_kind == "field":
        F = 1e-4 * rng.standard_normal(grid + (D,))
    elif force_kind == "uniform":
        # the reference casts a (D,) force to float32 (lbm.py:929-931)
        F = np.array([2e-4, -1e-4, 5e-5][:D], dtype=np.float32).astype(np.float64)
    else:
        F = None
    a = 1e-3 * rng.standard_normal(grid)               # weights on density
    b = 1e-3 * rng.standard_normal(grid + (lat.Q,))    # weights on f
    return lat, wall, f0, F, a, b


def _loss(f, rho, u, a, b):
    return 0.5 * (rho * (u ** 2).sum(-1)).sum() + (a * rho).sum() + (b * f).sum()


@pytest.mark.parametrize("lattice,grid", [("D3Q19", (8, 6, 10)), ("D2Q9", (14, 11))])
@pytest.mark.parametrize("force_kind", ["field", "uniform", "none"])
@pytest.mark.parametrize("storage,tol", [("f64", 1e-9), ("f32", 1e-4)])
def test_adjoint_matches_autograd_of_restatement(lattice, grid, force_kind, storage, tol):
    from maddening_b200 import LBMNode
    lat, wall, f0, F, a, b = _case(lattice, grid, 3, force_kind)
    steps, K, tau = 25, 6, 0.7
    # autograd oracle (float64, CPU)
    f0_t = torch.tensor(f0, dtype=torch.float64, requires_grad=True)
    F_t = None if F is None else torch.tensor(F, dtype=torch.float64, requires_grad=True)
    F_use = F_t if F_t is not None else torch.zeros(grid + (lat.D,), dtype=torch.float64)
    f, rho, u = RT.rollout(f0_t, torch.as_tensor(wall), F_use, tau, lat, steps)
    L = _loss(f, rho, u, torch.as_tensor(a), torch.as_tensor(b))
    L.backward()
    # hand-written adjoint
    node = LBMNode("adj", 1.0, grid_shape=grid, viscosity=(tau - 0.5) / 3.0, lattice=lattice,
                   wall_mask=wall, storage=storage)
    dt = torch.float64 if storage == "f64" else torch.float32
    f0_g = torch.tensor(f0, dtype=dt, device="cuda", requires_grad=True)
    bi = {}
    F_g = None
    if F is not None:
        F_g = torch.tensor(F, dtype=dt, device="cuda", requires_grad=True)
        bi["body_force"] = F_g
    out = node.rollout({"f": f0_g, "wall_mask": node.initial_state()["wall_mask"]}, bi, steps,
                       checkpoint_every=K)
    Lg = _loss(out["f"].double(), out["density"].double(), out["velocity"].double(),
               torch.as_tensor(a, device="cuda"), torch.as_tensor(b, device="cuda"))
    Lg.backward()
    lg, lt = float(Lg.detach()), float(L.detach())
    assert abs(lg - lt) <= 1e-6 * abs(lt) + 1e-12
    e_f0 = R.rel_l2(f0_g.grad.cpu().numpy(), f0_t.grad.numpy())
    assert e_f0 <= tol, e_f0
    if F is not None:
        e_F = R.rel_l2(F_g.grad.cpu().numpy(), F_t.grad.numpy())
        assert e_F <= tol, e_F


def test_adjoint_fp64_vs_central_differences():
    from maddening_b200 import LBMNode
    grid, steps, tau = (12, 10, 14), 60, 0.7
    lat, wall, f0, F, _, _ = _case("D3Q19", grid, 5, "field")
    node = LBMNode("fd", 1.0, grid_shape=grid, viscosity=(tau - 0.5) / 3.0, wall_mask=wall,
                   storage="f64")
    wm = node.initial_state()["wall_mask"]
    f0_g = torch.tensor(f0, dtype=torch.float64, device="cuda")
    F_g = torch.tensor(F, dtype=torch.float64, device="cuda", requires_grad=True)
    out = node.rollout({"f": f0_g, "wall_mask": wm}, {"body_force": F_g}, steps)
    _kinetic(out).backward()
    grad = F_g.grad.cpu().numpy()
    rng = np.random.default_rng(9)
    for _ in range(8):
        idx = tuple(int(rng.integers(0, n)) for n in grid) + (int(rng.integers(0, 3)),)
        eps = 1e-3 * max(abs(F[idx]), 1e-4)
        vals = []
        for sgn in (1.0, -1.0):
            Fp = F.copy()
            Fp[idx] += sgn * eps
            o = node.run({"f": f0_g, "wall_mask": wm},
                         {"body_force": torch.tensor(Fp, device="cuda")}, steps)
            vals.append(float(_kinetic(o)))
        fd = (vals[0] - vals[1]) / (2 * eps)
        assert abs(fd - grad[idx]) <= 1e-6 * abs(grad[idx]) + 1e-20, (idx, fd, grad[idx])


def test_differentiated_rollout_128cube_1000_steps():
    """The differentiated-rollout configuration at full size."""
    from maddening_b200 import LBMNode
    grid, steps, tau, K = (128, 128, 128), 1000, 0.7, 32
    rng = np.random.default_rng(0)
    F = 1e-6 * rng.standard_normal(grid + (3,))
    wall = R.z_walls(grid)
    node32 = LBMNode("c3", 1.0, grid_shape=grid, viscosity=(tau - 0.5) / 3.0, wall_mask=wall)
    node64 = LBMNode("c3", 1.0, grid_shape=grid, viscosity=(tau - 0.5) / 3.0, wall_mask=wall,
                     storage="f64")
    st = node32.initial_state()
    F32 = torch.tensor(F, dtype=torch.float32, device="cuda", requires_grad=True)
    out = node32.rollout(st, {"body_force": F32}, steps, checkpoint_every=K)
    _kinetic(out).backward()
    grad = F32.grad.double().cpu().numpy()
    st64 = node64.initial_state()
    F64 = torch.tensor(F, dtype=torch.float64, device="cuda")
    cells = [tuple(int(rng.integers(0, n)) for n in grid) for _ in range(16)]
    errs = []
    for cell in cells:
        wall_cell = bool(wall[cell])
        comp = int(rng.integers(0, 3))
        idx = cell + (comp,)
        eps = 1e-3 * max(abs(F[idx]), 1e-6)  # 1e-3 relative to the force scale
        vals = []
        for sgn in (1.0, -1.0):
            Fp = F64.clone()
            Fp[idx] += sgn * eps
            vals.append(float(_kinetic(node64.run(st64, {"body_force": Fp}, steps))))
        fd = (vals[0] - vals[1]) / (2 * eps)
        errs.append(abs(grad[idx] - fd) / max(abs(fd), 1e-30))
        assert errs[-1] <= 1e-4, (idx, wall_cell, grad[idx], fd)
    print(f"\n128^3 x 1000 steps, checkpoint 32: FP32 adjoint vs FP64 central differences, "
          f"max rel err over 16 cells = {max(errs):.2e}")
