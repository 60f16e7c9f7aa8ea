"""Pin the LBMPipeNode oracle (``oracle/lbm_pipe_ref.py``) to the reference's
own ``src/maddening/nodes/lbm_pipe.py`` executed by ``tests/golden/make_golden.py``
(single phase and Shan-Chen multiphase): masks and initial state equal, x64
steps bit-exact, float32 steps within float32 rounding."""

import numpy as np
import pytest

from oracle import lbm_pipe_ref as P
from tests.golden.make_golden import PIPE_CASES

KEYS = ("f", "density", "velocity", "tracer", "tracer_f")


def _oracle(case, mode):
    kw = {k: v for k, v in case.items() if k not in ("name", "steps", "bi", "scale_block")}
    return P.OraclePipe(mode=mode, **kw)


def _initial(node, case):
    """The case's starting state: the initial state, with the populations of
    one block scaled down where the case asks for it."""
    st = node.initial_state()
    if "scale_block" in case:
        (a0, a1), (b0, b1), (c0, c1), factor = case["scale_block"]
        f = st["f"].copy()
        f[a0:a1, b0:b1, c0:c1] *= np.float32(factor)
        st["f"] = f
    return st


@pytest.mark.parametrize("case", PIPE_CASES, ids=[c["name"] for c in PIPE_CASES])
def test_masks_and_initial_state(golden, case):
    p = f"{case['name']}|x64|"
    node = _oracle(case, "x64")
    np.testing.assert_array_equal(node.wall, golden[p + "wall"])
    np.testing.assert_array_equal(node.prop, golden[p + "propeller"])
    st = _initial(node, case)
    for key in KEYS:
        np.testing.assert_array_equal(st[key], golden[p + key + "0"])


@pytest.mark.parametrize("case", PIPE_CASES, ids=[c["name"] for c in PIPE_CASES])
def test_pipe_x64_bit_exact(golden, case):
    p = f"{case['name']}|x64|"
    node = _oracle(case, "x64")
    st = {k: v.astype(np.float64) for k, v in _initial(node, case).items()}
    st = node.update(st, case["bi"])
    for key in KEYS:
        np.testing.assert_array_equal(st[key], golden[p + "step1_" + key])
    st = node.run(st, case["bi"], case["steps"] - 1)
    for key in KEYS:
        np.testing.assert_array_equal(st[key], golden[p + "final_" + key])


@pytest.mark.parametrize("case", PIPE_CASES, ids=[c["name"] for c in PIPE_CASES])
def test_pipe_f32_within_rounding(golden, case):
    p = f"{case['name']}|f32|"
    node = _oracle(case, "f32")
    st = node.run(_initial(node, case), case["bi"], case["steps"])
    for key in KEYS:
        assert st[key].dtype == np.float32
        np.testing.assert_allclose(st[key], golden[p + "final_" + key], rtol=0,
                                   atol=8 * np.finfo(np.float32).eps)


def test_multiphase_case_reaches_floor_and_clamp():
    """The floor case really rescales populations and clamps the shifted velocity."""
    case = next(c for c in PIPE_CASES if c["name"] == "pipe_multiphase_floor_and_clamp")
    node = _oracle(case, "x64")
    st = {k: v.astype(np.float64) for k, v in _initial(node, case).items()}
    density, u = P.macroscopic(st["f"])
    force = P.shan_chen_force(density, node.G, node.rho_0, node.wall, node.rho_wall)
    u_shift = u + force / np.maximum(density, 0.01)[..., None]
    assert np.sqrt((u_shift ** 2).sum(-1)).max() > 0.25
    out = node.update(st, case["bi"])
    assert (out["density"] == 0.01).any()
