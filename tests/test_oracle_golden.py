"""Pin the CPU oracle to the reference's own executed code.

The fixtures in ``tests/golden/lbm_golden.npz`` come from running the
reference's ``src/maddening/nodes/lbm.py`` unmodified (see
``tests/golden/make_golden.py``).  The FP64 ("x64") oracle must reproduce
them to the last bit; the float32 mode within float32 rounding.
"""

import numpy as np
import pytest

from oracle import lbm_ref as R
from tests.golden.make_golden import CASES


def _oracle_for(golden, case, mode):
    p = f"{case['name']}|{mode}|"
    wall = golden[p + "wall"]
    node = R.OracleLBM(case["grid"], case["viscosity"], case["lattice"],
                       wall_mask=wall if wall.any() else None,
                       inlet_face=case["faces"][0], outlet_face=case["faces"][1],
                       mode=mode)
    st = node.initial_state()
    f0 = golden[p + "f0"]
    st["f"] = f0.astype(np.float64) if mode == "x64" else f0
    bi = {}
    for k in golden.files:
        if k.startswith(p + "bi_"):
            name = k[len(p) + 3:]
            v = golden[k]
            bi[name] = np.float32(v) if v.ndim == 0 else v
    return node, st, bi, p


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_x64_bit_exact(golden, case):
    node, st, bi, p = _oracle_for(golden, case, "x64")
    st = node.update(st, bi)
    for key in ("f", "density", "velocity", "pressure"):
        np.testing.assert_array_equal(st[key], golden[p + "step1_" + key])
    for _ in range(case["steps"] - 1):
        st = node.update(st, bi)
    for key in ("f", "density", "velocity", "pressure"):
        assert st[key].dtype == golden[p + "final_" + key].dtype
        np.testing.assert_array_equal(st[key], golden[p + "final_" + key])
    flux = node.compute_boundary_fluxes(st)
    np.testing.assert_allclose(flux["outlet_pressure_avg"],
                               golden[p + "final_outlet_pressure_avg"], rtol=1e-12)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_f32_within_rounding(golden, case):
    node, st, bi, p = _oracle_for(golden, case, "f32")
    for _ in range(case["steps"]):
        st = node.update(st, bi)
    for key in ("f", "density", "velocity", "pressure"):
        ref = golden[p + "final_" + key]
        assert st[key].dtype == np.float32
        np.testing.assert_allclose(st[key], ref, rtol=0, atol=4 * np.finfo(np.float32).eps)


def test_unit_kernels_match_reference(golden):
    for lat in (R.d3q19(), R.d2q9()):
        t = "unit_" + lat.name.lower()
        np.testing.assert_array_equal(lat.e, golden[t + "_e"])
        np.testing.assert_array_equal(lat.w, golden[t + "_w"])
        np.testing.assert_array_equal(lat.opp, golden[t + "_opp"])
        np.testing.assert_array_equal(lat.opp, golden[t + "_opp_map"])
        rho, u, F, f = (golden[t + k] for k in ("_rho", "_u", "_F", "_frand"))
        np.testing.assert_array_equal(R.equilibrium(rho, u, lat), golden[t + "_feq"])
        d, v = R.macroscopic(f, lat, F)
        np.testing.assert_array_equal(d, golden[t + "_macro_rho"])
        np.testing.assert_array_equal(v, golden[t + "_macro_u"])
        np.testing.assert_array_equal(R.stream(f, lat), golden[t + "_stream"])
        np.testing.assert_allclose(R.guo_forcing(rho, u, F, 0.73, lat),
                                   golden[t + "_guo"], rtol=0, atol=1e-18)
        for axis in range(lat.D):
            for side in ("min", "max"):
                g = golden[f"{t}_classify_{axis}_{side}"]
                nk, nu, nt = g[:3]
                k, un, tg = R.classify_directions(lat.e, axis, side)
                assert list(g[3:3 + nk]) == k
                assert list(g[3 + nk:3 + nk + nu]) == un
                assert list(g[3 + nk + nu:]) == tg
