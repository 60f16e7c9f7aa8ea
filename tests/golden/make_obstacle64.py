"""Golden FP64 run of the obstacle flow at 64^3 (seeded synthetic input).

The benchmark workload's physics on a lattice the NumPy oracle finishes in
minutes: 64x64x64 D3Q19, seeded sphere obstacles
(maddening_b200.geometry.random_spheres(grid, seed=0): radii 4-12, 10 % solid,
centres kept 16 cells off the x faces), velocity inlet u = (0.05, 0, 0) at
x_min, zero-gradient outlet at x_max, periodic in y and z, tau = 0.6
(viscosity 0.1 / 3), initial state rho = 1, u = 0, f = f_eq (the node's
initial_state); then 500 steps of the FP64 oracle and of the float32 oracle
(the reference's own float32 arithmetic).

The velocity inlet and the zero-gradient outlet are extensions with no
reference counterpart: this fixture pins the GPU kernels to the oracle's
restatement of them, not to the reference.

Writes tests/golden/obstacle64.npz: the wall mask's packed bits (a check
that the generator still gives this geometry), the FP64 run's rho - 1 and u
after 500 steps (float32 copies: 6e-8 relative rounding, far below the 1e-5
bound) and the float32 path's relative L2 errors against it.  Takes about ten
minutes (single-threaded NumPy).
"""

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from maddening_b200.geometry import random_spheres  # noqa: E402
from oracle import lbm_ref as R  # noqa: E402

N, STEPS, SEED, U_IN = 64, 500, 0, 0.05


def main():
    grid = (N, N, N)
    wall = random_spheres(grid, seed=SEED)
    bi = {"inlet_velocity": np.array([U_IN, 0.0, 0.0])}
    out = {"wall_bits": np.packbits(wall.reshape(-1))}
    res = {}
    for mode in ("x64", "f32"):
        node = R.OracleLBM(grid, 0.1 / 3.0, "D3Q19", wall_mask=wall,
                           outlet_condition="zero_gradient", mode=mode)
        st = node.initial_state()
        if mode == "x64":
            st["f"] = st["f"].astype(np.float64)
        t0 = time.time()
        for _ in range(STEPS):
            st = node.update(st, bi)
        print(f"{mode}: {STEPS} steps in {time.time() - t0:.1f} s", flush=True)
        rd = np.sum(st["f"].astype(np.float64), axis=-1) - 1.0
        res[mode] = (rd, st["density"].astype(np.float64), st["velocity"].astype(np.float64))
    out["x64_rho_dev"] = res["x64"][0].astype(np.float32)
    out["x64_u"] = res["x64"][2].astype(np.float32)
    out["f32_relL2_rho"] = np.float64(R.rel_l2(res["f32"][1], res["x64"][1]))
    out["f32_relL2_u"] = np.float64(R.rel_l2(res["f32"][2], res["x64"][2]))
    out["f32_relL2_rho_dev"] = np.float64(R.rel_l2(res["f32"][0], res["x64"][0]))
    print({k: float(v) for k, v in out.items() if k.startswith("f32_")})
    np.savez_compressed(Path(__file__).with_name("obstacle64.npz"), **out)


if __name__ == "__main__":
    main()
