"""Lattice <-> SI transforms (``maddening_b200/transforms.py``) against the
reference's own ``core/transforms_unit.py`` executed by
``tests/golden/make_golden.py``: same values and names; and on torch tensors."""

import numpy as np
import pytest
import torch

from maddening_b200 import transforms as T
from tests.golden.make_golden import TRANSFORM_SCALES

NAMES = ("lbm_to_si_force", "si_to_lbm_force", "lbm_to_si_torque", "lbm_to_si_velocity",
         "lbm_to_si_pressure", "lbm_to_si_length")


def _make(name, dx, dt, rho):
    fn = getattr(T, name)
    if name == "lbm_to_si_velocity":
        return fn(dx, dt)
    if name == "lbm_to_si_length":
        return fn(dx)
    return fn(dx, dt, rho)


@pytest.mark.parametrize("i", range(len(TRANSFORM_SCALES)))
@pytest.mark.parametrize("name", NAMES)
def test_matches_reference(golden, i, name):
    fn = _make(name, *TRANSFORM_SCALES[i])
    x = golden["transform|input"]
    np.testing.assert_array_equal(fn(x), golden[f"transform|{i}|{name}|values"])
    assert fn.__qualname__ == str(golden[f"transform|{i}|{name}|qualname"])


def test_force_round_trip_and_tensors():
    dx, dt, rho = 1e-3, 1e-6, 1060.0
    to_si, to_lbm = T.lbm_to_si_force(dx, dt, rho), T.si_to_lbm_force(dx, dt, rho)
    f = torch.tensor([1e-6, -2e-5, 3e-4], dtype=torch.float64, requires_grad=True)
    back = to_lbm(to_si(f))
    torch.testing.assert_close(back, f, rtol=1e-15, atol=0)
    back.sum().backward()
    torch.testing.assert_close(f.grad, torch.ones(3, dtype=torch.float64), rtol=1e-15, atol=0)
