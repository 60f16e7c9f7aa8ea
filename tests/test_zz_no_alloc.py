"""Allocation-free variant of the reference step: ``lbm_update_noalloc``.

Some callers of this library cannot allocate device memory or hand over a
workspace: a custom-call handler whose runtime gives it no scratch allocator,
an embedded or real-time loop where device allocation is not allowed.
``lbm_update_noalloc`` serves them: its scratch is a static device array inside
the library (``LBM_NOALLOC_SCRATCH_BYTES`` = 24 MiB, held by every GPU that
loads the library until the process exits), so the call itself allocates
nothing.  The GPU test calls it through the C ABI and checks it against
``lbm_update`` with a caller-provided workspace on two calls in a row: the
second call starts with the static array still holding the first call's data.
This file is named so that pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest

from maddening_b200 import _lib



def _fill_args(lattice, grid, storage, rng, torch):
    dev = "cuda"
    D = len(grid)
    dt = torch.float64 if storage == "f64" else torch.float32
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12) if lattice == 19 else \
        np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    f0 = w * (1.0 + 1e-3 * rng.standard_normal(grid + (lattice,)))
    f0 = torch.as_tensor(f0.astype(np.float32).astype(np.float64), device=dev).to(dt)
    wall = torch.as_tensor((rng.random(grid) < 0.15).astype(np.uint8), device=dev)
    force = torch.as_tensor(1e-4 * rng.standard_normal(grid + (D,)), device=dev).to(dt)
    a = _lib.lbm_step_args()
    a.force_mode = _lib.FORCE_FIELD
    a.force_field = force.data_ptr()
    a.wall = wall.data_ptr()
    a.inlet.kind, a.inlet.face = _lib.BC_PRESSURE, _lib.FACES["x_min"]
    a.inlet.value[0] = 1.004
    a.outlet.kind, a.outlet.face = _lib.BC_PRESSURE, _lib.FACES["x_max"]
    a.outlet.value[0] = 1.0
    return f0, a, (wall, force), dt


def _outputs(grid, lattice, dt, torch):
    D = len(grid)
    f = torch.empty(grid + (lattice,), dtype=dt, device="cuda")
    rho = torch.empty(grid, dtype=dt, device="cuda")
    u = torch.empty(grid + (D,), dtype=dt, device="cuda")
    p = torch.empty(grid, dtype=dt, device="cuda")
    m = _lib.lbm_moments()
    m.density, m.velocity, m.pressure = rho.data_ptr(), u.data_ptr(), p.data_ptr()
    return (f, rho, u, p), m


@pytest.mark.gpu
@pytest.mark.parametrize("lattice,grid,storage", [
    (19, (24, 20, 32), "f32"),   # one-pass kernel: the array holds its status word
    (19, (24, 20, 30), "f32"),   # rows of 30 cells: two passes through the array
    (19, (24, 20, 30), "f16"),
    (9, (40, 36), "f64"),
    (19, (69, 69, 69), "f32"),   # 24.97 MB of the 25.17 MB array, two passes
])
def test_noalloc_matches_workspace_update_on_two_calls(lattice, grid, storage):
    import torch
    rng = np.random.default_rng(11)
    plan = _lib.Plan(lattice, grid, 0.8, storage)
    lib = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    f0, args, keep, dt = _fill_args(lattice, grid, storage, rng, torch)
    ws = torch.empty(plan.workspace_bytes(), dtype=torch.uint8, device="cuda")

    ref_in, got_in = f0, f0
    for call in range(2):
        ref, m_ref = _outputs(grid, lattice, dt, torch)
        _lib.check(lib.lbm_update(plan.handle, stream, ref_in.data_ptr(), ref[0].data_ptr(),
                                  C.byref(args), C.byref(m_ref), ws.data_ptr(), ws.numel()))
        got, m_got = _outputs(grid, lattice, dt, torch)
        _lib.check(lib.lbm_update_noalloc(plan.handle, stream, got_in.data_ptr(),
                                          got[0].data_ptr(), C.byref(args), C.byref(m_got)))
        torch.cuda.synchronize()
        # the same kernels in the same order on the same inputs: equal bit for bit
        for g, r in zip(got, ref):
            assert torch.equal(g, r), call
        ref_in, got_in = ref[0], got[0]
    del keep


@pytest.mark.parametrize("grid", [(128, 128, 128), (70, 70, 68)])
def test_noalloc_rejects_lattices_beyond_the_static_scratch(grid):
    """A lattice whose populations need more than the 24 MiB array (128^3: 159
    MB; 70 x 70 x 68: 25.3 MB, just over) is rejected before any device work,
    with a message naming the limit."""
    plan = _lib.Plan(19, grid, 0.8, "f32")
    assert plan.state_bytes() > _lib.NOALLOC_SCRATCH_BYTES
    args = _lib.lbm_step_args()
    fake = C.c_void_p(0x1000)  # never dereferenced: the size check comes first
    rc = _lib.lib().lbm_update_noalloc(plan.handle, None, fake, fake, C.byref(args), None)
    assert rc == -4
    msg = _lib.last_error()
    assert "static array" in msg and str(_lib.NOALLOC_SCRATCH_BYTES) in msg
