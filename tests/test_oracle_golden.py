"""Pin the CPU oracle to the reference's own executed code.

The fixtures in ``tests/golden/lbm_golden.npz`` come from running the
reference's ``src/maddening/nodes/lbm.py`` unmodified (see
``tests/golden/make_golden.py``).  The FP64 ("x64") oracle must reproduce
them to the last bit; the float32 mode within float32 rounding.
"""

import numpy as np
import pytest

from oracle import lbm_ref as R
from tests.golden.make_golden import CASES, PADDED_CASES


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


def test_stream_padded_matches_reference(golden):
    for lat in (R.d3q19(), R.d2q9()):
        t = "unit_" + lat.name.lower()
        np.testing.assert_array_equal(R.stream_padded(golden[t + "_fpad"], lat, 1),
                                      golden[t + "_stream_padded"])


def _padded_inputs(golden, case, mode):
    p = f"{case['name']}|{mode}|"
    node = R.OracleLBM(case["grid"], case["viscosity"], case["lattice"],
                       inlet_face=case["faces"][0], outlet_face=case["faces"][1], mode=mode)
    f_pad = golden[p + "f_pad"]
    st = {"f": f_pad.astype(np.float64) if mode == "x64" else f_pad,
          "density": golden[p + "density_pad"], "velocity": golden[p + "velocity_pad"],
          "pressure": golden[p + "pressure_pad"], "wall_mask": golden[p + "wall_pad"]}
    bi = {}
    for k in golden.files:
        if k.startswith(p + "bi_"):
            v = golden[k]
            bi[k[len(p) + 3:]] = np.float32(v) if v.ndim == 0 else v
    return node, st, bi, p


@pytest.mark.parametrize("case", PADDED_CASES, ids=[c["name"] for c in PADDED_CASES])
def test_oracle_update_padded_x64_bit_exact(golden, case):
    node, st, bi, p = _padded_inputs(golden, case, "x64")
    out = node.update_padded(st, bi)
    for key in ("f", "density", "velocity", "pressure"):
        ref = golden[p + "out_" + key]
        assert out[key].dtype == ref.dtype, key
        np.testing.assert_array_equal(out[key], ref)


@pytest.mark.parametrize("case", PADDED_CASES, ids=[c["name"] for c in PADDED_CASES])
def test_oracle_update_padded_f32_within_rounding(golden, case):
    node, st, bi, p = _padded_inputs(golden, case, "f32")
    out = node.update_padded(st, bi)
    for key in ("f", "density", "velocity", "pressure"):
        np.testing.assert_allclose(out[key], golden[p + "out_" + key], rtol=0,
                                   atol=4 * np.finfo(np.float32).eps)


def test_update_padded_of_periodic_pad_equals_update():
    """The reference's own check (tests/nodes/test_lbm_stream_padded.py:66-186):
    a periodic pad on every axis makes update_padded's interior equal update."""
    lat = R.d3q19()
    grid = (6, 5, 7)
    rng = np.random.default_rng(4)
    wall = rng.random(grid) < 0.15
    wall[0] = wall[-1] = False
    node = R.OracleLBM(grid, 0.1, "D3Q19", wall_mask=wall)
    st = node.initial_state()
    st["f"] = lat.w * (1 + 1e-3 * rng.standard_normal(grid + (19,)))
    bi = {"inlet_pressure": np.float32(1 / 3 + 1e-3), "outlet_pressure": np.float32(1 / 3),
          "body_force": 1e-5 * rng.standard_normal(grid + (3,))}
    ref = node.update(st, bi)
    pad = lambda a, extra=0: np.pad(a, [(1, 1)] * 3 + [(0, 0)] * extra, mode="wrap")
    stp = {"f": pad(st["f"], 1), "density": pad(st["density"]),
           "velocity": pad(st["velocity"], 1), "pressure": pad(st["pressure"]),
           "wall_mask": pad(st["wall_mask"])}
    # an interior-shaped force field is zero-padded (lbm.py:826-832); pad it
    # periodically here so the halo cells collide with their own force
    bi_p = dict(bi, body_force=pad(bi["body_force"], 1))
    out = node.update_padded(stp, bi_p)
    inner = (slice(1, -1),) * 3
    # equal up to the summation order of NumPy's matrix products (which
    # depends on the array shape): 1e-15
    for key in ("f", "density", "velocity", "pressure"):
        np.testing.assert_allclose(out[key][inner], ref[key].astype(out[key].dtype),
                                   rtol=0, atol=1e-15)
