"""LBMPipeNode on the GPU (``lbm_pipe_rollout``) against the reference's own
``LBMPipeNode`` executed on the golden cases (single phase and Shan-Chen
multiphase): initial state equal, one step and the full case within float32
rounding of the x64 run (FP32 storage), within 1e-7 (FP64 storage: the
reference's float32 lattice weights are its own rounding of 1/18 and 1/36),
per-step ``update`` equal to the fused ``run``; and the CPU oracle on larger
pipes over 100 steps."""

import numpy as np
import pytest
import torch

from oracle import lbm_pipe_ref as P
from tests.golden.make_golden import PIPE_CASES

pytestmark = pytest.mark.gpu

KEYS = ("f", "density", "velocity", "tracer", "tracer_f")
F32_EPS = float(np.finfo(np.float32).eps)


def _node(case, storage="f32"):
    from maddening_b200.pipe import LBMPipeNode
    kw = {k: v for k, v in case.items() if k not in ("name", "steps", "bi", "scale_block")}
    return LBMPipeNode(case["name"], 1.0, storage=storage, **kw)


def _start(node, case):
    """The initial state, with the populations of one block scaled down where
    the case asks for it (in float32, as the fixtures were made)."""
    st = node.initial_state()
    if "scale_block" in case:
        (a0, a1), (b0, b1), (c0, c1), factor = case["scale_block"]
        f = st["f"].to(torch.float32).clone()
        f[a0:a1, b0:b1, c0:c1] *= np.float32(factor)
        st = dict(st, f=f.to(st["f"].dtype))
    return st


def _np(t):
    return t.detach().cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("case", PIPE_CASES, ids=[c["name"] for c in PIPE_CASES])
def test_initial_state_equals_reference(golden, case):
    node = _node(case)
    st = _start(node, case)
    p = f"{case['name']}|x64|"
    for key in KEYS:
        np.testing.assert_array_equal(st[key].cpu().numpy(), golden[p + key + "0"])


@pytest.mark.parametrize("case", PIPE_CASES, ids=[c["name"] for c in PIPE_CASES])
def test_pipe_steps_match_reference(golden, case):
    node = _node(case)
    p = f"{case['name']}|x64|"
    st = _start(node, case)
    one = node.update(st, case["bi"], 1.0)
    # single phase keeps normalised offsets (f - w) / w on the device, so the
    # error of a step is a fraction of an ulp of the deviations; multiphase
    # keeps the populations themselves in FP32: a step's density is a sum of
    # 19 rounded populations, a few ulp of the field's magnitude
    mp = case.get("G", 0.0) != 0.0
    for key in KEYS:
        ref = golden[p + "step1_" + key]
        tol = 8 * F32_EPS * max(1.0, np.abs(ref).max()) if mp else 4e-7
        err = np.max(np.abs(_np(one[key]) - ref))
        assert err <= tol, (key, err)
    out = node.run(st, case["bi"], case["steps"])
    for key in KEYS:
        ref = golden[p + "final_" + key]
        tol = 24 * F32_EPS * max(1.0, np.abs(ref).max()) if mp else 1e-6
        err = np.max(np.abs(_np(out[key]) - ref))
        assert err <= tol, (key, err)
    # single phase: per-step updates equal the fused rollout only up to the
    # float32 state between steps (the fused run keeps offsets on the
    # device); multiphase keeps the populations themselves, bit for bit
    cur = st
    for _ in range(case["steps"]):
        cur = node.update(cur, case["bi"], 1.0)
    tol = 0.0 if case.get("G", 0.0) != 0.0 else 1e-6
    for key in KEYS:
        assert np.max(np.abs(_np(cur[key]) - _np(out[key]))) <= tol, key


@pytest.mark.parametrize("case", PIPE_CASES, ids=[c["name"] for c in PIPE_CASES])
def test_pipe_fp64_storage(golden, case):
    node = _node(case, "f64")
    p = f"{case['name']}|x64|"
    st = _start(node, case)
    out = node.run(st, case["bi"], case["steps"])
    assert out["f"].dtype == torch.float64
    # against the reference: apart from FP64 rounding, the kernel differs
    # through the reference's float32 lattice weights (their sum 1 + 1.49e-8
    # moves the mass of a cell by omega rho 1.49e-8 per step)
    for key in KEYS:
        ref = golden[p + "final_" + key]
        err = np.max(np.abs(_np(out[key]) - ref))
        assert err <= 2e-7 * max(1.0, np.abs(ref).max()), (key, err)
    # against the oracle with the weights 1/3, 1/18, 1/36: FP64 rounding only
    kw = {k: v for k, v in case.items() if k not in ("name", "steps", "bi", "scale_block")}
    orc = P.OraclePipe(mode="x64", weights="exact", **kw)
    ref = orc.run({k: _np(v) for k, v in st.items()}, case["bi"], case["steps"])
    for key in KEYS:
        err = np.max(np.abs(_np(out[key]) - ref[key]))
        assert err <= 1e-12, (key, err)


def test_pipe_100_steps_against_oracle():
    """A 48 x 20 x 18 pipe, partly filled, propeller + gravity, 100 steps: the
    FP32 kernel against the FP64 oracle."""
    kw = dict(nx=48, ny=20, nz=18, tau=0.75, pipe_radius=0.9, propeller_x=12,
              propeller_radius=0.8, propeller_strength=4e-4, initial_velocity=0.005,
              gravity=1e-5, fill_fraction=0.7, tau_tracer=0.65)
    from maddening_b200.pipe import LBMPipeNode
    node = LBMPipeNode("p", 1.0, **kw)
    out = node.run(node.initial_state(), {}, 100)
    orc = P.OraclePipe(mode="x64", **kw)
    st = {k: v.astype(np.float64) for k, v in orc.initial_state().items()}
    ref = orc.run(st, {}, 100)
    # density: the reference's float32 lattice weights sum to 1 + 1.49e-8, so its
    # collision changes the mass by omega * 1.49e-8 per step (2e-6 after 100
    # steps here); the kernel's weights are exact
    for key, tol in (("velocity", 1e-4), ("density", 5e-6), ("tracer", 1e-5)):
        rel = np.linalg.norm(_np(out[key]) - ref[key]) / np.linalg.norm(ref[key])
        assert rel <= tol, (key, rel)


@pytest.mark.parametrize("storage,weights,tol", [("f32", "reference", 1e-5),
                                                  ("f64", "exact", 1e-11)])
def test_multiphase_100_steps_against_oracle(storage, weights, tol):
    """A 40 x 18 x 20 pipe half filled with liquid (G = -4.5), propeller and
    gravity, 100 steps, against the FP64 oracle: FP32 storage against the
    reference's arithmetic; FP64 storage against the same arithmetic with the
    weights 1/3, 1/18, 1/36 (with the reference's float32 weights the two
    differ by 3.3e-6 in velocity after 100 steps, the weights' own effect)."""
    kw = dict(nx=40, ny=18, nz=20, tau=0.8, pipe_radius=0.9, propeller_x=8,
              propeller_radius=0.8, propeller_strength=4e-4, initial_velocity=0.005,
              gravity=-1e-5, fill_fraction=0.5, tau_tracer=0.6, G=-4.5, rho_liquid=1.3,
              rho_gas=0.3)
    from maddening_b200.pipe import LBMPipeNode
    node = LBMPipeNode("p", 1.0, storage=storage, **kw)
    out = node.run(node.initial_state(), {}, 100)
    orc = P.OraclePipe(mode="x64", weights=weights, **kw)
    st = {k: v.astype(np.float64) for k, v in orc.initial_state().items()}
    ref = orc.run(st, {}, 100)
    errs = {}
    for key in ("velocity", "density", "tracer", "f"):
        errs[key] = np.linalg.norm(_np(out[key]) - ref[key]) / np.linalg.norm(ref[key])
    assert max(errs.values()) <= tol, errs
