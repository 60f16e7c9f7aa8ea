"""Golden wall masks from the reference's own voxelizer.

Executes the unmodified ``src/maddening/nodes/lbm_geometry.py`` of the
reference (``voxelize_vessel``, lbm_geometry.py:17-142) under the NumPy
stand-in for the ``jax`` API subset that make_golden.py installs (JAX is not
installed here), for a few grids and vessel parameter sets, and writes the
masks' packed bits to tests/golden/geometry_golden.npz.

    python tests/golden/make_geometry.py <reference checkout root>

The root may also come from the environment variable MADDENING_REF_ROOT.
"""

import importlib
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import make_golden  # noqa: E402

CASES = [
    # the reference's own test parameters (tests/nodes/test_lbm.py:460-492)
    ((64, 32, 32), dict(parent_radius=6.0, daughter_radius=4.0, parent_length=30.0,
                        daughter_length=25.0, bifurcation_angle=30.0)),
    ((48, 40, 24), dict(parent_radius=5.5, daughter_radius=3.25, parent_length=20.0,
                        daughter_length=30.0, bifurcation_angle=45.0)),
    ((33, 17, 21), dict(parent_radius=4.0, daughter_radius=4.0, parent_length=0.0,
                        daughter_length=40.0, bifurcation_angle=12.5)),
    ((40, 31, 16), dict(parent_radius=7.0, daughter_radius=2.5, parent_length=39.0,
                        daughter_length=0.0, bifurcation_angle=60.0)),
]


def main(ref_root=None):
    ref_root = ref_root or os.environ.get("MADDENING_REF_ROOT")
    if not ref_root:
        sys.exit("usage: make_geometry.py <reference root> (or set MADDENING_REF_ROOT)")
    make_golden._install_shims(Path(ref_root))
    geo = importlib.import_module("maddening.nodes.lbm_geometry")
    out = {}
    for i, (grid, params) in enumerate(CASES):
        mask = np.asarray(make_golden._plain(geo.voxelize_vessel(grid, params)))
        assert mask.dtype == np.bool_ and mask.shape == grid
        out[f"vessel{i}_grid"] = np.array(grid, dtype=np.int64)
        out[f"vessel{i}_params"] = np.frombuffer(json.dumps(params).encode(), dtype=np.uint8)
        out[f"vessel{i}_bits"] = np.packbits(mask.reshape(-1))
        print(f"vessel{i} {grid}: {mask.mean():.4f} wall")
    np.savez_compressed(HERE / "geometry_golden.npz", **out)


if __name__ == "__main__":
    main(*sys.argv[1:])
