"""The torch restatement (autograd oracle) equals the NumPy oracle's FP64 forward."""

import numpy as np
import torch

from oracle import lbm_ref as R
from oracle import lbm_ref_torch as RT


def test_torch_restatement_matches_numpy_oracle():
    for lattice, grid in (("D3Q19", (6, 5, 7)), ("D2Q9", (9, 8))):
        rng = np.random.default_rng(2)
        lat = R.lattice(lattice)
        wall = rng.random(grid) < 0.2
        f0 = lat.w * (1 + 1e-3 * rng.standard_normal(grid + (lat.Q,)))
        F = 1e-4 * rng.standard_normal(grid + (lat.D,))
        orc = R.OracleLBM(grid, 0.1, lattice, wall_mask=wall)
        st = orc.initial_state()
        st["f"] = f0
        st = orc.run(st, {"body_force": F}, 5)
        f, rho, u = RT.rollout(torch.tensor(f0), torch.as_tensor(wall), torch.tensor(F),
                               orc.tau, lat, 5, checkpoint=False)
        np.testing.assert_allclose(f.numpy(), st["f"], rtol=0, atol=1e-15)
        np.testing.assert_allclose(rho.numpy(), st["density"], rtol=0, atol=1e-14)
        np.testing.assert_allclose(u.numpy(), st["velocity"], rtol=0, atol=1e-15)


def test_torch_restatement_gradcheck_tiny():
    lat = R.d2q9()
    rng = np.random.default_rng(4)
    grid = (4, 3)
    wall = torch.as_tensor(rng.random(grid) < 0.3)
    f0 = torch.tensor(lat.w * (1 + 1e-2 * rng.standard_normal(grid + (9,))))
    F = torch.tensor(1e-2 * rng.standard_normal(grid + (2,)), requires_grad=True)

    def fn(F):
        _, rho, u = RT.rollout(f0, wall, F, 0.8, lat, 3, checkpoint=False)
        return (rho * (u ** 2).sum(-1)).sum()

    assert torch.autograd.gradcheck(fn, (F,), eps=1e-6, atol=1e-9)
