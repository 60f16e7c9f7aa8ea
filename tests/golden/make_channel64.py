"""Golden FP64 run of the 64^3 force-driven channel (seeded synthetic input).

Lattice 64x64x64 D3Q19, walls on the first and last z plane, periodic x/y,
tau = 0.8 (viscosity 0.1), uniform body force (1e-6, 0, 0) given as float32,
rho0 = 1 + 1e-3 N(0,1) from numpy.random.default_rng(0), u0 = 0,
f0 = f_eq(rho0, 0) rounded to float32 (the reference's state dtype); then 500
steps of the FP64 oracle (the reference under jax_enable_x64) and of the
float32 oracle (the reference's default float32 path).

Writes tests/golden/channel64.npz with the FP64 run's rho - 1 and u after 500
steps (float32 copies: their 6e-8 relative rounding is far below the 1e-5
parity bound) and the float32 path's relative L2 errors against it.
Takes a few minutes (single-threaded NumPy).
"""

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import lbm_ref as R  # noqa: E402

N, STEPS, SEED = 64, 500, 0


def main():
    lat = R.d3q19()
    grid = (N, N, N)
    f0, _ = R.channel_state(lat, grid, seed=SEED)
    bi = {"body_force": np.array([1e-6, 0.0, 0.0], dtype=np.float32)}
    out = {"f0_check": f0[:2, :2, :2].copy()}
    res = {}
    for mode in ("x64", "f32"):
        node = R.OracleLBM(grid, 0.1, "D3Q19", wall_mask=R.z_walls(grid), mode=mode)
        st = node.initial_state()
        st["f"] = f0.astype(np.float64) if mode == "x64" else f0.copy()
        t0 = time.time()
        for i in range(STEPS):
            st = node.update(st, bi)
        print(f"{mode}: {STEPS} steps in {time.time() - t0:.1f} s", flush=True)
        rd = np.sum(st["f"].astype(np.float64), axis=-1) - 1.0
        res[mode] = (rd, st["density"].astype(np.float64), st["velocity"].astype(np.float64))
    out["x64_rho_dev"] = res["x64"][0].astype(np.float32)
    out["x64_u"] = res["x64"][2].astype(np.float32)
    # error of the reference's own float32 path against FP64 (informational)
    out["f32_relL2_rho"] = np.float64(R.rel_l2(res["f32"][1], res["x64"][1]))
    out["f32_relL2_u"] = np.float64(R.rel_l2(res["f32"][2], res["x64"][2]))
    out["f32_relL2_rho_dev"] = np.float64(R.rel_l2(res["f32"][0], res["x64"][0]))
    np.savez_compressed(Path(__file__).with_name("channel64.npz"), **out)


if __name__ == "__main__":
    main()
