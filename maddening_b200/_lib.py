"""ctypes binding of ``liblbm_b200.so`` (the C ABI in ``include/lbm_b200.h``).

The library must be built in-tree (``python -m maddening_b200.build``); a
missing library raises immediately -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "liblbm_b200.so"

LBM_OK = 0
STATUS = {0: "LBM_OK", -1: "LBM_ERR_INVALID", -2: "LBM_ERR_UNSUPPORTED",
          -3: "LBM_ERR_CUDA", -4: "LBM_ERR_WORKSPACE", -5: "LBM_ERR_TIMEOUT"}

LBM_D2Q9, LBM_D3Q19 = 9, 19
STORAGE = {"f32": 0, "f16": 1, "bf16": 2, "f64": 3}
FORCE_NONE, FORCE_UNIFORM, FORCE_FIELD = 0, 1, 2
FACES = {"x_min": 0, "x_max": 1, "y_min": 2, "y_max": 3, "z_min": 4, "z_max": 5}
BC_NONE, BC_PRESSURE, BC_VELOCITY, BC_ZERO_GRADIENT = 0, 1, 2, 3
MOMENTS_DENSITY_DEVIATION = 1
NOALLOC_SCRATCH_BYTES = 24 << 20  # LBM_NOALLOC_SCRATCH_BYTES


class LbmError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


PLAN_SINGLE_CELLS = 2
PLAN_PAIRED_CELLS = 4
PLAN_TWO_PASS = 8
PLAN_TEST_WAIT_TIMEOUT = 16


class lbm_desc(C.Structure):
    _fields_ = [("lattice", C.c_int32), ("storage", C.c_int32),
                ("shape", C.c_int64 * 3), ("tau", C.c_double), ("flags", C.c_uint32)]


class lbm_face_bc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("face", C.c_int32), ("value", C.c_double * 3)]


class lbm_step_args(C.Structure):
    _fields_ = [("force_mode", C.c_int32), ("force", C.c_double * 3),
                ("force_field", C.c_void_p), ("wall", C.c_void_p),
                ("inlet", lbm_face_bc), ("outlet", lbm_face_bc),
                ("dev_values", C.c_void_p)]


class lbm_moments(C.Structure):
    _fields_ = [("density", C.c_void_p), ("velocity", C.c_void_p),
                ("pressure", C.c_void_p), ("flags", C.c_uint32)]


class lbm_history(C.Structure):
    _fields_ = [("f", C.c_void_p), ("density", C.c_void_p), ("velocity", C.c_void_p),
                ("pressure", C.c_void_p)]


_P = C.c_void_p
_SIGS = {
    "lbm_abi_version": ([], C.c_int),
    "lbm_last_error": ([C.c_char_p, C.c_size_t], C.c_int),
    "lbm_plan_create": ([C.POINTER(lbm_desc), C.POINTER(_P)], C.c_int),
    "lbm_plan_destroy": ([_P], C.c_int),
    "lbm_state_bytes": ([_P, C.POINTER(C.c_size_t)], C.c_int),
    "lbm_workspace_bytes": ([_P, C.POINTER(C.c_size_t)], C.c_int),
    "lbm_equilibrium": ([_P, _P, _P, _P, _P], C.c_int),
    "lbm_update": ([_P, _P, _P, _P, C.POINTER(lbm_step_args), C.POINTER(lbm_moments),
                    _P, C.c_size_t], C.c_int),
    "lbm_rollout": ([_P, _P, _P, _P, C.c_int64, C.POINTER(lbm_step_args),
                     C.POINTER(lbm_moments), _P, C.c_size_t], C.c_int),
    "lbm_update_noalloc": ([_P, _P, _P, _P, C.POINTER(lbm_step_args),
                            C.POINTER(lbm_moments)], C.c_int),
    "lbm_update_padded": ([_P, _P, _P, _P, C.POINTER(lbm_step_args), C.POINTER(lbm_moments),
                           _P, C.c_size_t], C.c_int),
    "lbm_rollout_history": ([_P, _P, _P, _P, C.c_int64, C.c_int64, C.POINTER(lbm_step_args),
                             C.POINTER(lbm_moments), C.POINTER(lbm_history), _P, C.c_size_t],
                            C.c_int),
    "lbm_adjoint_workspace_bytes": ([_P, C.c_int64, C.c_int64, C.POINTER(C.c_size_t)],
                                    C.c_int),
    "lbm_rollout_forward": ([_P, _P, _P, _P, C.c_int64, C.c_int64, C.POINTER(lbm_step_args),
                             C.POINTER(lbm_moments), _P, C.c_size_t], C.c_int),
    "lbm_rollout_backward": ([_P, _P, _P, C.c_int64, C.c_int64, C.POINTER(lbm_step_args),
                              _P, _P, _P, _P, _P, _P, C.c_size_t], C.c_int),
    "lbm_reduce_workspace_bytes": ([_P, C.POINTER(C.c_size_t)], C.c_int),
    "lbm_state_from_f": ([_P, _P, _P, _P, C.POINTER(lbm_step_args), C.c_int64], C.c_int),
    "lbm_state_step": ([_P, _P, _P, _P, C.POINTER(lbm_step_args), C.c_int64, C.c_int64,
                        C.c_int64], C.c_int),
    "lbm_state_to_f": ([_P, _P, _P, _P, C.POINTER(lbm_step_args), C.POINTER(lbm_moments)],
                       C.c_int),
    "lbm_mass_momentum": ([_P, _P, _P, _P, _P, C.c_size_t], C.c_int),
}

_lock = threading.Lock()
_lib = None


def lib() -> C.CDLL:
    """Load the library once; raise if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m maddening_b200.build` "
                    "(the LBM step has no CPU fallback)")
            h = C.CDLL(os.fspath(LIB_PATH))
            for name, (args, res) in _SIGS.items():
                fn = getattr(h, name)
                fn.argtypes = args
                fn.restype = res
            if h.lbm_abi_version() != 1:
                raise ImportError("liblbm_b200.so ABI version mismatch")
            _lib = h
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().lbm_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != LBM_OK:
        raise LbmError(status, last_error())


class Plan:
    """Owns one ``lbm_plan`` (immutable lattice/shape/tau/storage)."""

    def __init__(self, q: int, shape, tau: float, storage: str = "f32", flags: int = 0):
        d = lbm_desc()
        d.lattice = q
        d.storage = STORAGE[storage]
        d.flags = int(flags)
        for i, n in enumerate(tuple(shape)[:3]):
            d.shape[i] = int(n)
        d.tau = float(tau)
        h = _P()
        check(lib().lbm_plan_create(C.byref(d), C.byref(h)))
        self._h = h
        self.q = q
        self.shape = tuple(int(n) for n in shape)
        self.tau = float(tau)
        self.storage = storage
        self.flags = int(flags)

    @property
    def handle(self):
        return self._h

    def _size(self, fn) -> int:
        n = C.c_size_t()
        check(fn(self._h, C.byref(n)))
        return int(n.value)

    def state_bytes(self) -> int:
        return self._size(lib().lbm_state_bytes)

    def workspace_bytes(self) -> int:
        return self._size(lib().lbm_workspace_bytes)

    def reduce_workspace_bytes(self) -> int:
        return self._size(lib().lbm_reduce_workspace_bytes)

    def adjoint_workspace_bytes(self, n_steps: int, checkpoint_every: int = 0) -> int:
        n = C.c_size_t()
        check(lib().lbm_adjoint_workspace_bytes(self._h, int(n_steps), int(checkpoint_every),
                                                C.byref(n)))
        return int(n.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.lbm_plan_destroy(h)
            self._h = None
