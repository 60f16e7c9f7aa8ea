"""Pin the LBMPipeNode oracle (``oracle/lbm_pipe_ref.py``) to the reference's
own ``src/maddening/nodes/lbm_pipe.py`` executed by ``tests/golden/make_golden.py``
(single-phase mode): masks and initial state equal, x64 steps bit-exact,
float32 steps within float32 rounding."""

import numpy as np
import pytest

from oracle import lbm_pipe_ref as P
from tests.golden.make_golden import PIPE_CASES

KEYS = ("f", "density", "velocity", "tracer", "tracer_f")


def _oracle(case, mode):
    kw = {k: v for k, v in case.items() if k not in ("name", "steps", "bi")}
    return P.OraclePipe(mode=mode, **kw)


@pytest.mark.parametrize("case", PIPE_CASES, ids=[c["name"] for c in PIPE_CASES])
def test_masks_and_initial_state(golden, case):
    p = f"{case['name']}|x64|"
    node = _oracle(case, "x64")
    np.testing.assert_array_equal(node.wall, golden[p + "wall"])
    np.testing.assert_array_equal(node.prop, golden[p + "propeller"])
    st = node.initial_state()
    for key in KEYS:
        np.testing.assert_array_equal(st[key], golden[p + key + "0"])


@pytest.mark.parametrize("case", PIPE_CASES, ids=[c["name"] for c in PIPE_CASES])
def test_pipe_x64_bit_exact(golden, case):
    p = f"{case['name']}|x64|"
    node = _oracle(case, "x64")
    st = {k: v.astype(np.float64) for k, v in node.initial_state().items()}
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
    st = node.run(node.initial_state(), case["bi"], case["steps"])
    for key in KEYS:
        assert st[key].dtype == np.float32
        np.testing.assert_allclose(st[key], golden[p + "final_" + key], rtol=0,
                                   atol=8 * np.finfo(np.float32).eps)
