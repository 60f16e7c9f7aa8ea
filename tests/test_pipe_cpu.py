"""LBMPipeNode host side (no GPU): the reference's validation, masks and
contract surface (src/maddening/nodes/lbm_pipe.py:493-662), masks and the
multiphase initial density checked against the reference-executed golden
fixtures."""

import numpy as np
import pytest

from maddening_b200.pipe import LBMPipeNode
from tests.golden.make_golden import PIPE_CASES


def _kw(case):
    return {k: v for k, v in case.items() if k not in ("name", "steps", "bi", "scale_block")}


@pytest.mark.parametrize("case", PIPE_CASES, ids=[c["name"] for c in PIPE_CASES])
def test_masks_match_reference(golden, case):
    node = LBMPipeNode(case["name"], 1.0, **_kw(case))
    p = f"{case['name']}|x64|"
    np.testing.assert_array_equal(node.wall_mask, golden[p + "wall"])
    np.testing.assert_array_equal(node.propeller_mask, golden[p + "propeller"])


@pytest.mark.parametrize("kw,msg", [(dict(tau=0.5), "tau must be > 0.5"),
                                    (dict(tau_tracer=0.4), "tau_tracer must be > 0.5"),
                                    (dict(fill_fraction=0.0), "fill_fraction"),
                                    (dict(G=-4.5, rho_liquid=0.2, rho_gas=0.25), "rho_liquid"),
                                    (dict(G=-4.5, rho_gas=0.0), "rho_gas must be > 0"),
                                    (dict(G=-4.5, rho_0=0.0), "rho_0 must be > 0")])
def test_validation_like_reference(kw, msg):
    with pytest.raises(ValueError, match=msg):
        LBMPipeNode("p", 1.0, nx=8, ny=8, nz=8, **kw)


MP_CASES = [c for c in PIPE_CASES if c.get("G", 0.0) != 0.0]


@pytest.mark.parametrize("case", MP_CASES, ids=[c["name"] for c in MP_CASES])
def test_multiphase_initial_density_matches_reference(golden, case):
    node = LBMPipeNode(case["name"], 1.0, **_kw(case))
    np.testing.assert_array_equal(node._multiphase_density(),
                                  golden[f"{case['name']}|x64|density0"])


def test_multiphase_parameters():
    node = LBMPipeNode("p", 1.0, nx=8, ny=8, nz=8, G=-4.5, rho_liquid=1.2, rho_gas=0.3)
    assert node.params["G"] == -4.5
    assert node.params["rho_wall"] == 1.2
    node = LBMPipeNode("p", 1.0, nx=8, ny=8, nz=8, G=-4.5, rho_wall=0.4)
    assert node.params["rho_wall"] == 0.4


def test_contract_surface():
    node = LBMPipeNode("p", 0.01, nx=16, ny=10, nz=12, tau=0.9)
    assert node.halo_width() == {0: 1, 1: 1, 2: 1}
    assert node.viscosity == pytest.approx((0.9 - 0.5) / 3)
    assert node.params["propeller_strength"] == 0.0005
    assert node.params["rho_wall"] == node.params["rho_liquid"]
    assert node.meta.algorithm_id == "MADD-NODE-006"
    with pytest.raises(NotImplementedError):
        node.derivatives({}, {})
