"""C-ABI checks that need no GPU: exports, struct layouts, host validation."""

import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from maddening_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lbm_b200.h")


def _declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^int\s+(lbm_\w+)\s*\(", src, flags=re.M)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.lib()
    names = _declared_functions()
    assert len(names) >= 10
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\s[TW]\s(lbm_\w+)$", out, flags=re.M))
    missing = [n for n in names if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for n in names:
        assert hasattr(lib, n)
    assert lib.lbm_abi_version() == 1


def test_struct_layout_matches_header():
    prog = r"""
    #include <stdio.h>
    #include <stddef.h>
    #include "lbm_b200.h"
    int main(void) {
      printf("%zu %zu %zu %zu\n", sizeof(lbm_desc), sizeof(lbm_face_bc),
             sizeof(lbm_step_args), sizeof(lbm_moments));
      printf("%zu %zu %zu %zu %zu %zu\n", offsetof(lbm_step_args, force),
             offsetof(lbm_step_args, force_field), offsetof(lbm_step_args, wall),
             offsetof(lbm_step_args, inlet), offsetof(lbm_step_args, outlet),
             offsetof(lbm_step_args, dev_values));
      printf("%zu %zu %zu\n", offsetof(lbm_desc, shape), offsetof(lbm_desc, tau),
             offsetof(lbm_desc, flags));
      return 0;
    }
    """
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in lines[0].split()]
    assert sizes == [C.sizeof(_lib.lbm_desc), C.sizeof(_lib.lbm_face_bc),
                     C.sizeof(_lib.lbm_step_args), C.sizeof(_lib.lbm_moments)]
    offs = [int(x) for x in lines[1].split()]
    S = _lib.lbm_step_args
    assert offs == [S.force.offset, S.force_field.offset, S.wall.offset, S.inlet.offset,
                    S.outlet.offset, S.dev_values.offset]
    doffs = [int(x) for x in lines[2].split()]
    assert doffs == [_lib.lbm_desc.shape.offset, _lib.lbm_desc.tau.offset,
                     _lib.lbm_desc.flags.offset]


@pytest.mark.parametrize("q,shape,tau,msg", [
    (19, (8, 8, 8), 0.5, "tau must be > 0.5"),
    (19, (8, 8, 8), 0.2, "tau must be > 0.5"),
    (7, (8, 8, 8), 0.8, "Unknown lattice"),
    (19, (8, 0, 8), 0.8, "out of range"),
])
def test_plan_validation(q, shape, tau, msg):
    with pytest.raises(_lib.LbmError, match=msg) as ei:
        _lib.Plan(q, shape, tau)
    assert ei.value.status == -1


def test_plan_sizes():
    p = _lib.Plan(19, (16, 12, 8), 0.8)
    n = 16 * 12 * 8
    assert p.state_bytes() == 19 * n * 4
    sb = (19 * n * 4 + 255) // 256 * 256
    assert p.workspace_bytes() == 2 * sb + 256  # two population copies + status word
    p16 = _lib.Plan(19, (16, 12, 8), 0.8, "f16")
    assert p16.state_bytes() == 19 * n * 2
    p64 = _lib.Plan(9, (16, 12), 0.8, "f64")
    assert p64.state_bytes() == 9 * 16 * 12 * 8


def test_update_rejects_missing_workspace_before_any_device_work():
    p = _lib.Plan(19, (8, 8, 8), 0.8)
    lib = _lib.lib()
    args = _lib.lbm_step_args()
    fake = C.c_void_p(0x1000)  # never dereferenced: validation fails first
    rc = lib.lbm_update(p.handle, None, fake, fake, C.byref(args), None, None, 0)
    assert rc == -4
    assert "workspace" in _lib.last_error()
    rc = lib.lbm_rollout(p.handle, None, fake, fake, 0, C.byref(args), None, fake, 1 << 30)
    assert rc == -1
    assert "n_steps" in _lib.last_error()
    rc = lib.lbm_update(p.handle, None, None, fake, C.byref(args), None, fake, 1 << 30)
    assert rc == -1


def test_update_padded_rejects_blocks_without_a_halo_before_any_device_work():
    lib = _lib.lib()
    args = _lib.lbm_step_args()
    fake = C.c_void_p(0x1000)  # never dereferenced: validation fails first
    thin = _lib.Plan(19, (8, 2, 8), 0.8)
    rc = lib.lbm_update_padded(thin.handle, None, fake, fake, C.byref(args), None, fake, 1 << 30)
    assert rc == -1 and "halo" in _lib.last_error()
    p = _lib.Plan(19, (8, 8, 8), 0.8)
    rc = lib.lbm_update_padded(p.handle, None, fake, fake, C.byref(args), None, fake, 16)
    assert rc == -4 and "workspace" in _lib.last_error()
    args.outlet.kind, args.outlet.face = _lib.BC_ZERO_GRADIENT, _lib.FACES["x_max"]
    short = _lib.Plan(19, (4, 8, 8), 0.8)
    rc = lib.lbm_update_padded(short.handle, None, fake, fake, C.byref(args), None, fake,
                               1 << 30)
    assert rc == -1 and "interior" in _lib.last_error()


def test_plan_rejects_unknown_and_reserved_flags():
    from maddening_b200 import _lib
    for flags in (1, 32, 64, 1 << 30):
        with pytest.raises(_lib.LbmError, match="reserved plan flags"):
            _lib.Plan(19, (8, 8, 8), 0.8, "f32", flags=flags)
    _lib.Plan(19, (8, 8, 8), 0.8, "f32", flags=_lib.PLAN_TWO_PASS | _lib.PLAN_SINGLE_CELLS)
