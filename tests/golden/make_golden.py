"""Generate golden vectors by executing the reference's own ``lbm.py``.

JAX is not installed in this container (and has no offline wheel), so the
reference module ``maddening.nodes.lbm`` cannot be imported as shipped.  This
script executes that unmodified source file against a small NumPy-backed
stand-in for the ``jax`` API subset it uses (``jnp.roll/stack/where/sum/...``
and functional ``x.at[idx].set(v)`` updates).  Two arithmetic modes are
emulated:

* ``x64``: NumPy float64 constants promote float32 arrays -- the reference
  under ``jax_enable_x64`` (the FP64 oracle the build is graded against).
* ``f32``: float64 NumPy constants are demoted to float32 whenever they meet
  a stand-in array -- JAX's default canonicalisation (informational only:
  XLA may order float32 roundings differently).

The package ``__init__`` files of ``maddening.core`` and ``maddening.nodes``
import JAX-heavy siblings; they are bypassed by registering bare package
modules whose ``__path__`` points at the real directories, so only
``core/node.py``, ``core/compliance/*`` and ``nodes/lbm.py`` execute.

Run from the repository root (needs the reference checkout)::

    python tests/golden/make_golden.py [/path/to/reference]

It rewrites ``tests/golden/lbm_golden.npz``.  The fixtures are committed;
nothing at test time reads the reference.
"""

from __future__ import annotations

import importlib
import os
import sys
import types
from pathlib import Path

import numpy as np

MODE = {"value": "x64"}


# ---------------------------------------------------------------------------
# NumPy-backed stand-in for the jax API subset used by nodes/lbm.py
# ---------------------------------------------------------------------------


class JArray(np.ndarray):
    """ndarray with JAX's functional ``.at[idx].set(v)`` update."""

    @property
    def at(self):
        return _At(self)

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        conv = []
        for x in inputs:
            if isinstance(x, JArray):
                x = x.view(np.ndarray)
            elif MODE["value"] == "f32" and isinstance(x, np.ndarray) \
                    and x.dtype == np.float64:
                x = x.astype(np.float32)
            conv.append(x)
        if "out" in kwargs:
            kwargs["out"] = tuple(o.view(np.ndarray) if isinstance(o, JArray) else o
                                  for o in kwargs["out"])
        res = getattr(ufunc, method)(*conv, **kwargs)
        return _wrap(res)


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIdx(self.arr, idx)


class _AtIdx:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def set(self, value):
        out = np.array(self.arr, copy=True)
        out[self.idx] = np.asarray(value)
        return out.view(JArray)


def _wrap(x):
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, np.ndarray):
        if MODE["value"] == "f32" and x.dtype == np.float64:
            x = x.astype(np.float32)
        return x.view(JArray)
    return x


def _plain(x):
    return x.view(np.ndarray) if isinstance(x, JArray) else x


def _make_jnp():
    jnp = types.ModuleType("jax.numpy")
    for name in ("float32", "float64", "int32", "uint8", "bool_"):
        setattr(jnp, name, getattr(np, name))

    def asarray(x, dtype=None):
        a = np.asarray(_plain(x), dtype=dtype)
        return _wrap(np.array(a, copy=True))

    def zeros(shape, dtype=None):
        return _wrap(np.zeros(shape, dtype=dtype if dtype is not None else np.float32))

    def ones(shape, dtype=None):
        return _wrap(np.ones(shape, dtype=dtype if dtype is not None else np.float32))

    jnp.asarray = asarray
    jnp.array = asarray
    jnp.zeros = zeros
    jnp.ones = ones
    jnp.zeros_like = lambda x, dtype=None: _wrap(np.zeros_like(_plain(x), dtype=dtype))
    jnp.full_like = lambda x, v, dtype=None: _wrap(np.full_like(_plain(x), _plain(v), dtype=dtype))
    jnp.sum = lambda x, axis=None, keepdims=False: _wrap(np.sum(_plain(x), axis=axis, keepdims=keepdims))
    jnp.maximum = lambda a, b: _wrap(np.maximum(_plain(a), _plain(b)))
    jnp.roll = lambda x, s, axis=None: _wrap(np.roll(_plain(x), s, axis=axis))
    jnp.stack = lambda xs, axis=0: _wrap(np.stack([_plain(v) for v in xs], axis=axis))
    jnp.where = lambda c, a, b: _wrap(np.where(_plain(c), _plain(a), _plain(b)))
    jnp.broadcast_to = lambda x, shape: _wrap(np.broadcast_to(_plain(x), shape))
    jnp.pad = lambda x, w: _wrap(np.pad(_plain(x), w))
    jnp.arange = lambda *a, dtype=None: _wrap(np.arange(*a, dtype=dtype))
    jnp.meshgrid = lambda *xs, indexing="xy": tuple(
        _wrap(np.array(m)) for m in np.meshgrid(*[_plain(x) for x in xs], indexing=indexing))
    jnp.sqrt = lambda x: _wrap(np.sqrt(_plain(x)))
    jnp.exp = lambda x: _wrap(np.exp(_plain(x)))
    jnp.tanh = lambda x: _wrap(np.tanh(_plain(x)))
    jnp.clip = lambda x, lo, hi: _wrap(np.clip(_plain(x), lo, hi))
    jnp.minimum = lambda a, b: _wrap(np.minimum(_plain(a), _plain(b)))
    jnp.all = lambda x: bool(np.all(_plain(x)))
    jnp.isfinite = lambda x: _wrap(np.isfinite(_plain(x)))
    jnp.ndarray = JArray
    return jnp


def _install_shims(ref_root: Path):
    jax = types.ModuleType("jax")
    jnp = _make_jnp()
    lax = types.ModuleType("jax.lax")

    def slice_in_dim(x, start, limit, axis=0):
        sl = [slice(None)] * np.ndim(x)
        sl[axis] = slice(start, limit)
        return _wrap(np.asarray(_plain(x))[tuple(sl)])

    lax.slice_in_dim = slice_in_dim
    jax.numpy = jnp
    jax.lax = lax
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp
    sys.modules["jax.lax"] = lax

    src = ref_root / "src"
    sys.path.insert(0, str(src))
    import maddening  # noqa: F401  (lazy __init__, no jax import)
    for pkg in ("maddening.core", "maddening.nodes", "maddening.api"):
        mod = types.ModuleType(pkg)
        mod.__path__ = [str(src / Path(*pkg.split(".")))]
        sys.modules[pkg] = mod
    return importlib.import_module("maddening.nodes.lbm")


# ---------------------------------------------------------------------------
# Cases
# ---------------------------------------------------------------------------


def _perturbed_f(lbm, node, seed, amp=1e-3):
    st = node.initial_state()
    f = np.asarray(_plain(st["f"]), dtype=np.float64)
    w = node._lat.w
    rng = np.random.default_rng(seed)
    f = f + amp * w * rng.standard_normal(f.shape)
    return f.astype(np.float32)          # float32-exact initial values


CASES = [
    # name, lattice, grid, viscosity, wall kind, inlet, outlet, bi kind, steps
    dict(name="d3q19_periodic_uniform_force", lattice="D3Q19", grid=(6, 5, 7),
         viscosity=0.1, walls=None, faces=("x_min", "x_max"),
         bi=dict(body_force="uniform"), steps=4),
    dict(name="d3q19_zwalls_uniform_force", lattice="D3Q19", grid=(5, 6, 8),
         viscosity=0.1, walls="z", faces=("x_min", "x_max"),
         bi=dict(body_force="uniform"), steps=4),
    dict(name="d3q19_random_walls_field_force", lattice="D3Q19", grid=(6, 7, 5),
         viscosity=0.05, walls="random", faces=("x_min", "x_max"),
         bi=dict(body_force="field"), steps=3),
    dict(name="d3q19_zou_he_x", lattice="D3Q19", grid=(8, 4, 6),
         viscosity=0.1, walls="y", faces=("x_min", "x_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 * 1.01, outlet_pressure=1.0 / 3.0),
         steps=4),
    dict(name="d3q19_zou_he_y_min_z_max", lattice="D3Q19", grid=(5, 6, 7),
         viscosity=0.08, walls="random", faces=("y_min", "z_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 2e-3, outlet_pressure=1.0 / 3.0 - 1e-3,
                 body_force="uniform"), steps=3),
    dict(name="d3q19_zou_he_same_face", lattice="D3Q19", grid=(4, 5, 6),
         viscosity=0.1, walls=None, faces=("z_max", "z_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 1e-3, outlet_pressure=1.0 / 3.0),
         steps=2),
    dict(name="d3q19_wall_mask_update", lattice="D3Q19", grid=(6, 5, 5),
         viscosity=0.1, walls="z", faces=("x_min", "x_max"),
         bi=dict(body_force="uniform", wall_mask_update="random"), steps=3),
    dict(name="d2q9_periodic_uniform_force", lattice="D2Q9", grid=(7, 6),
         viscosity=0.1, walls=None, faces=("x_min", "x_max"),
         bi=dict(body_force="uniform"), steps=5),
    dict(name="d2q9_channel_zou_he", lattice="D2Q9", grid=(12, 8),
         viscosity=0.1, walls="y2", faces=("x_min", "x_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 * 1.01, outlet_pressure=1.0 / 3.0),
         steps=5),
    dict(name="d2q9_zou_he_y_max_x_min_field", lattice="D2Q9", grid=(9, 7),
         viscosity=0.07, walls="random", faces=("y_max", "x_min"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 1e-3, outlet_pressure=1.0 / 3.0,
                 body_force="field"), steps=4),
    # last-axis extents that are multiples of 4 (vectorised kernels), with
    # rows of one vector, rows longer than a warp, and faces on that axis
    dict(name="d3q19_vec_faces_on_last_axis", lattice="D3Q19", grid=(4, 5, 12),
         viscosity=0.1, walls="random", faces=("z_min", "z_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 1e-3, outlet_pressure=1.0 / 3.0,
                 body_force="field"), steps=3),
    dict(name="d3q19_vec_long_rows", lattice="D3Q19", grid=(3, 3, 136),
         viscosity=0.1, walls="random", faces=("x_min", "y_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 1e-3, outlet_pressure=1.0 / 3.0,
                 body_force="uniform"), steps=3),
    dict(name="d3q19_vec_rows_of_4", lattice="D3Q19", grid=(6, 5, 4),
         viscosity=0.12, walls="z", faces=("z_min", "x_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 1e-3, outlet_pressure=1.0 / 3.0),
         steps=3),
    dict(name="d2q9_vec_long_rows", lattice="D2Q9", grid=(5, 132),
         viscosity=0.1, walls="random", faces=("y_min", "y_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 1e-3, outlet_pressure=1.0 / 3.0,
                 body_force="field"), steps=4),
    dict(name="d2q9_vec_rows_of_4", lattice="D2Q9", grid=(7, 4),
         viscosity=0.1, walls=None, faces=("x_min", "y_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 1e-3, body_force="uniform"), steps=3),
]


def _walls(kind, grid, rng):
    if kind is None:
        return None
    w = np.zeros(grid, dtype=bool)
    if kind == "z":
        w[..., 0] = True
        w[..., -1] = True
    elif kind == "y":
        w[:, 0, ...] = True
        w[:, -1, ...] = True
    elif kind == "y2":
        w[:, 0] = True
        w[:, -1] = True
    elif kind == "random":
        w = rng.random(grid) < 0.2
    return w


def run_case(lbm, jnp, case, mode, seed):
    rng = np.random.default_rng(seed + 1000)
    grid = case["grid"]
    D = len(grid)
    walls = _walls(case["walls"], grid, rng)
    node = lbm.LBMNode(name=case["name"], timestep=1.0, grid_shape=grid,
                       viscosity=case["viscosity"], lattice=case["lattice"],
                       wall_mask=walls, inlet_face=case["faces"][0],
                       outlet_face=case["faces"][1])
    f0 = _perturbed_f(lbm, node, seed)
    state = node.initial_state()
    f_in = f0.astype(np.float64) if mode == "x64" else f0
    state = {**state, "f": jnp.asarray(f_in)}
    bi, bi_np = {}, {}
    for k, v in case["bi"].items():
        if k == "body_force":
            if v == "uniform":
                arr = (np.array([1e-4, -3e-5, 2e-5][:D], dtype=np.float32))
            else:
                arr = (1e-4 * rng.standard_normal(grid + (D,))).astype(np.float32)
            bi[k] = jnp.asarray(arr)
            bi_np[k] = arr
        elif k == "wall_mask_update":
            arr = rng.random(grid) < 0.15
            bi[k] = jnp.asarray(arr)
            bi_np[k] = arr
        else:
            bi[k] = np.float32(v)
            bi_np[k] = np.float32(v)
    out = {"f0": f0, "wall": walls if walls is not None else np.zeros(grid, bool),
           "tau": np.float64(node.tau)}
    for k, v in bi_np.items():
        out["bi_" + k] = np.asarray(v)
    for step in range(case["steps"]):
        state = node.update(state, bi, 1.0)
        if step == 0:
            for key in ("f", "density", "velocity", "pressure"):
                out["step1_" + key] = np.asarray(_plain(state[key]))
    for key in ("f", "density", "velocity", "pressure"):
        out["final_" + key] = np.asarray(_plain(state[key]))
    flux = node.compute_boundary_fluxes(state, {}, 1.0)
    out["final_outlet_pressure_avg"] = np.asarray(_plain(flux["outlet_pressure_avg"]))
    return out


PADDED_CASES = [
    # update_padded (lbm.py:747-897) on a halo-padded state: the halo is a
    # periodic pad (what a single device gets) plus, for "foreign" halos, a
    # perturbation standing in for a neighbour shard's different data
    dict(name="padded_d3q19_walls_uniform_force", lattice="D3Q19", grid=(5, 4, 6),
         viscosity=0.1, walls="y", faces=("x_min", "x_max"),
         bi=dict(body_force="uniform"), halo="foreign"),
    dict(name="padded_d3q19_zou_he_field_force", lattice="D3Q19", grid=(6, 5, 4),
         viscosity=0.08, walls="random", faces=("x_min", "x_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 1e-3, outlet_pressure=1.0 / 3.0,
                 body_force="field"), halo="foreign"),
    dict(name="padded_d3q19_periodic_zou_he_z", lattice="D3Q19", grid=(4, 4, 7),
         viscosity=0.1, walls=None, faces=("z_min", "z_max"),
         bi=dict(inlet_pressure=1.0 / 3.0 + 1e-3, outlet_pressure=1.0 / 3.0),
         halo="periodic"),
    dict(name="padded_d2q9_walls_field_force", lattice="D2Q9", grid=(7, 6),
         viscosity=0.07, walls="random", faces=("y_min", "y_max"),
         bi=dict(body_force="field", inlet_pressure=1.0 / 3.0 + 1e-3), halo="foreign"),
]


def run_padded_case(lbm, jnp, case, mode, seed):
    """One update_padded call of the reference on a padded state."""
    rng = np.random.default_rng(seed + 2000)
    grid = case["grid"]
    D = len(grid)
    walls = _walls(case["walls"], grid, rng)
    node = lbm.LBMNode(name=case["name"], timestep=1.0, grid_shape=grid,
                       viscosity=case["viscosity"], lattice=case["lattice"],
                       wall_mask=walls, inlet_face=case["faces"][0],
                       outlet_face=case["faces"][1])
    f0 = _perturbed_f(lbm, node, seed)
    st = node.initial_state()
    pad = [(1, 1)] * D

    def pad_field(a, extra=0):
        return np.pad(np.asarray(_plain(a)), pad + [(0, 0)] * extra, mode="wrap")

    f_pad = pad_field(f0, 1)
    wall_pad = pad_field(np.asarray(_plain(st["wall_mask"])))
    if case["halo"] == "foreign":
        inner = tuple(slice(1, -1) for _ in range(D))
        halo_mask = np.ones(f_pad.shape[:D], dtype=bool)
        halo_mask[inner] = False
        w = node._lat.w
        noise = (1e-3 * w * rng.standard_normal(f_pad.shape)).astype(np.float32)
        f_pad = np.where(halo_mask[..., None], f_pad + noise, f_pad).astype(np.float32)
        wall_pad = np.where(halo_mask, rng.random(halo_mask.shape) < 0.3, wall_pad)
    wall_pad = wall_pad.astype(np.uint8)
    dens_pad = pad_field(st["density"])
    vel_pad = pad_field(st["velocity"], 1)
    prs_pad = pad_field(st["pressure"])
    f_in = f_pad.astype(np.float64) if mode == "x64" else f_pad
    state_p = {"f": jnp.asarray(f_in), "density": jnp.asarray(dens_pad),
               "velocity": jnp.asarray(vel_pad), "pressure": jnp.asarray(prs_pad),
               "wall_mask": jnp.asarray(wall_pad)}
    bi, bi_np = {}, {}
    for k, v in case["bi"].items():
        if k == "body_force":
            if v == "uniform":
                arr = np.array([1e-4, -3e-5, 2e-5][:D], dtype=np.float32)
            else:   # interior-shaped field: the reference zero-pads it
                arr = (1e-4 * rng.standard_normal(grid + (D,))).astype(np.float32)
            bi[k] = jnp.asarray(arr)
            bi_np[k] = arr
        else:
            bi[k] = np.float32(v)
            bi_np[k] = np.float32(v)
    out = {"f_pad": f_pad, "wall_pad": wall_pad, "density_pad": dens_pad,
           "velocity_pad": vel_pad, "pressure_pad": prs_pad, "tau": np.float64(node.tau)}
    for k, v in bi_np.items():
        out["bi_" + k] = np.asarray(v)
    res = node.update_padded(state_p, bi, 1.0)
    for key in ("f", "density", "velocity", "pressure"):
        out["out_" + key] = np.asarray(_plain(res[key]))
    return out


PIPE_CASES = [
    # LBMPipeNode (lbm_pipe.py:393-879), single phase
    dict(name="pipe_propeller_gravity_partial_fill", nx=12, ny=10, nz=10, tau=0.8,
         pipe_radius=0.9, propeller_x=3, propeller_radius=0.8, propeller_strength=5e-4,
         initial_velocity=0.01, gravity=2e-5, fill_fraction=0.6, tau_tracer=0.6, steps=4,
         bi={}),
    dict(name="pipe_odd_dims_force_override", nx=9, ny=11, nz=8, tau=0.7,
         pipe_radius=0.85, propeller_x=5, propeller_radius=0.7, propeller_strength=3e-4,
         initial_velocity=0.0, gravity=0.0, fill_fraction=1.0, tau_tracer=0.75, steps=3,
         bi={"propeller_force": 8e-4}),
    # multiphase (Shan-Chen pseudopotential with exact-difference forcing)
    dict(name="pipe_multiphase_partial_fill", nx=10, ny=10, nz=12, tau=0.9,
         pipe_radius=0.9, propeller_x=4, propeller_radius=0.8, propeller_strength=5e-4,
         initial_velocity=0.01, gravity=-1e-5, fill_fraction=0.5, tau_tracer=0.6, G=-4.5,
         rho_liquid=1.3, rho_gas=0.3, rho_0=1.0, steps=5, bi={}),
    dict(name="pipe_multiphase_odd_dims_rho_wall", nx=8, ny=9, nz=11, tau=0.75,
         pipe_radius=0.85, propeller_x=2, propeller_radius=0.7, propeller_strength=3e-4,
         initial_velocity=0.0, gravity=0.0, fill_fraction=1.0, tau_tracer=0.6, G=-4.2,
         rho_liquid=1.0, rho_gas=0.25, rho_0=1.0, rho_wall=0.5, steps=4,
         bi={"propeller_force": 8e-4}),
    # a near-empty block inside the liquid: the density floor rescales the
    # populations and the shifted velocity is clamped at its rim
    dict(name="pipe_multiphase_floor_and_clamp", nx=10, ny=10, nz=12, tau=0.8,
         pipe_radius=0.9, propeller_x=2, propeller_radius=0.8, propeller_strength=5e-4,
         initial_velocity=0.0, gravity=0.0, fill_fraction=1.0, tau_tracer=0.6, G=-6.0,
         rho_liquid=2.5, rho_gas=0.2, rho_0=1.0, steps=3, bi={},
         scale_block=((4, 7), (4, 7), (4, 7), 0.002)),
]


def run_pipe_case(pipe, jnp, case, mode):
    kw = {k: v for k, v in case.items() if k not in ("name", "steps", "bi", "scale_block")}
    node = pipe.LBMPipeNode(case["name"], 1.0, **kw)
    st = node.initial_state()
    if "scale_block" in case:
        (a0, a1), (b0, b1), (c0, c1), factor = case["scale_block"]
        f = np.array(np.asarray(_plain(st["f"])), dtype=np.float32)
        f[a0:a1, b0:b1, c0:c1] *= np.float32(factor)
        st = dict(st, f=jnp.asarray(f))
    out = {k + "0": np.asarray(_plain(v)) for k, v in st.items()}
    if mode == "x64":
        st = {k: jnp.asarray(np.asarray(_plain(v), dtype=np.float64)) for k, v in st.items()}
    bi = {k: v for k, v in case["bi"].items()}
    for step in range(case["steps"]):
        st = node.update(st, bi, 1.0)
        if step == 0:
            for key in ("f", "density", "velocity", "tracer", "tracer_f"):
                out["step1_" + key] = np.asarray(_plain(st[key]))
    for key in ("f", "density", "velocity", "tracer", "tracer_f"):
        out["final_" + key] = np.asarray(_plain(st[key]))
    out["wall"] = np.asarray(_plain(node._wall_mask))
    out["propeller"] = np.asarray(_plain(node._propeller_mask))
    return out


TRANSFORM_SCALES = [(1e-3, 1e-6, 1060.0), (2.5e-5, 3e-7, 998.2), (0.01, 0.02, 1.2)]


def transform_vectors(tu):
    """core/transforms_unit.py: each factory applied to a ramp, and its name."""
    x = np.linspace(-2.0, 3.0, 11)
    out = {}
    for i, (dx, dt, rho) in enumerate(TRANSFORM_SCALES):
        made = {"lbm_to_si_force": tu.lbm_to_si_force(dx, dt, rho),
                "si_to_lbm_force": tu.si_to_lbm_force(dx, dt, rho),
                "lbm_to_si_torque": tu.lbm_to_si_torque(dx, dt, rho),
                "lbm_to_si_velocity": tu.lbm_to_si_velocity(dx, dt),
                "lbm_to_si_pressure": tu.lbm_to_si_pressure(dx, dt, rho),
                "lbm_to_si_length": tu.lbm_to_si_length(dx)}
        for name, fn in made.items():
            out[f"transform|{i}|{name}|values"] = np.asarray(fn(x))
            out[f"transform|{i}|{name}|qualname"] = np.array(fn.__qualname__)
    out["transform|input"] = x
    return out


def frame_states():
    """States for the streaming-frame fixtures: the shape of the reference's
    own encoder test (scalars and a 20-cell rod) and a mixed-dtype lattice
    state (float32 populations, float64 density, float16 velocity, uint8 wall
    mask, int64 counter, Python scalar)."""
    rng = np.random.default_rng(11)
    grid = (4, 3, 5)
    return {
        "rods": {"ball": {"position": np.array(5.0, dtype=np.float32),
                          "velocity": np.array(-3.2, dtype=np.float32)},
                 "heat_rod": {"temperature": np.ones(20, dtype=np.float32) * 20.0},
                 "table": {"position": np.array(0.0, dtype=np.float32)}},
        "lattice": {"vessel": {"f": rng.random(grid + (19,)).astype(np.float32),
                               "density": 1.0 + 1e-3 * rng.standard_normal(grid),
                               "velocity": (0.05 * rng.standard_normal(grid + (3,))).astype(np.float16),
                               "wall_mask": (rng.random(grid) < 0.3).astype(np.uint8),
                               "steps": np.arange(6, dtype=np.int64) * 1000003},
                    "heart": {"pressure": np.array(13.25), "volume": 71.5}},
    }


FRAME_SUBSCRIPTIONS = {"all": None, "subset": {"vessel": ["velocity", "density", "nope"],
                                               "heart": ["volume"], "missing": ["x"]},
                       "nothing": {}}


def frame_vectors(be):
    """api/binary_encoder.py: schema and frame bytes of each state and subscription."""
    import json
    out = {}
    for sname, state in frame_states().items():
        for subname, sub in FRAME_SUBSCRIPTIONS.items():
            enc = be.BinaryStateEncoder(state, fields=sub)
            frame = enc.encode(0.125 * len(sname), state)
            key = f"frame|{sname}|{subname}"
            out[key + "|bytes"] = np.frombuffer(frame, dtype=np.uint8).copy()
            out[key + "|schema"] = np.array(json.dumps(enc.schema()))
    return out


def unit_vectors(lbm, jnp, seed=7):
    """Golden vectors for the pure kernels on random inputs (x64)."""
    rng = np.random.default_rng(seed)
    out = {}
    for lat in (lbm.d3q19(), lbm.d2q9()):
        tag = lat.name.lower()
        grid = (4, 3, 5)[: lat.D]
        rho = 1.0 + 0.01 * rng.standard_normal(grid)
        u = 0.05 * rng.standard_normal(grid + (lat.D,))
        F = 1e-3 * rng.standard_normal(grid + (lat.D,))
        f = rng.random(grid + (lat.Q,))
        out[f"{tag}_e"] = lat.e
        out[f"{tag}_w"] = lat.w
        out[f"{tag}_opp"] = lat.opp
        out[f"{tag}_rho"] = rho
        out[f"{tag}_u"] = u
        out[f"{tag}_F"] = F
        out[f"{tag}_frand"] = f
        out[f"{tag}_feq"] = np.asarray(_plain(lbm._equilibrium(jnp.asarray(rho), jnp.asarray(u), lat.e, lat.w, lat.cs2)))
        d, v = lbm._compute_macroscopic(jnp.asarray(f), lat.e, force=jnp.asarray(F))
        out[f"{tag}_macro_rho"] = np.asarray(_plain(d))
        out[f"{tag}_macro_u"] = np.asarray(_plain(v))
        out[f"{tag}_stream"] = np.asarray(_plain(lbm._stream(jnp.asarray(f), lat.e, lat.D)))
        fpad = np.random.default_rng(seed + lat.Q).random(tuple(n + 2 for n in grid) + (lat.Q,))
        out[f"{tag}_fpad"] = fpad
        out[f"{tag}_stream_padded"] = np.asarray(_plain(lbm._stream_padded(
            jnp.asarray(fpad), lat.e, lat.D, 1)))
        out[f"{tag}_guo"] = np.asarray(_plain(lbm._guo_forcing(
            jnp.asarray(rho), jnp.asarray(u), jnp.asarray(F), 0.73, lat.e, lat.w, lat.cs2)))
        out[f"{tag}_opp_map"] = lbm._get_opp_map(lat.e)
        for axis in range(lat.D):
            for side in ("min", "max"):
                k, un, t = lbm._classify_directions(lat.e, axis, side)
                out[f"{tag}_classify_{axis}_{side}"] = np.array(
                    [len(k), len(un), len(t)] + k + un + t, dtype=np.int32)
    return out


def main(ref_root=None):
    ref_root = ref_root or os.environ.get("MADDENING_REF_ROOT")
    if not ref_root:
        sys.exit("usage: make_golden.py <reference root> (or set MADDENING_REF_ROOT)")
    ref_root = Path(ref_root)
    lbm = _install_shims(ref_root)
    jnp = sys.modules["jax.numpy"]
    golden = {}
    MODE["value"] = "x64"
    golden.update({f"unit_{k}": v for k, v in unit_vectors(lbm, jnp).items()})
    for i, case in enumerate(CASES):
        for mode in ("x64", "f32"):
            MODE["value"] = mode
            res = run_case(lbm, jnp, case, mode, seed=i)
            for k, v in res.items():
                golden[f"{case['name']}|{mode}|{k}"] = v
    for i, case in enumerate(PADDED_CASES):
        for mode in ("x64", "f32"):
            MODE["value"] = mode
            res = run_padded_case(lbm, jnp, case, mode, seed=100 + i)
            for k, v in res.items():
                golden[f"{case['name']}|{mode}|{k}"] = v
    pipe = importlib.import_module("maddening.nodes.lbm_pipe")
    for case in PIPE_CASES:
        for mode in ("x64", "f32"):
            MODE["value"] = mode
            res = run_pipe_case(pipe, jnp, case, mode)
            for k, v in res.items():
                golden[f"{case['name']}|{mode}|{k}"] = v
    MODE["value"] = "x64"
    golden.update(transform_vectors(importlib.import_module("maddening.core.transforms_unit")))
    golden.update(frame_vectors(importlib.import_module("maddening.api.binary_encoder")))
    out = Path(__file__).with_name("lbm_golden.npz")
    np.savez_compressed(out, **golden)
    meta = {c["name"]: c for c in CASES + PADDED_CASES + PIPE_CASES}
    print(f"wrote {out} ({out.stat().st_size / 1024:.1f} KiB, {len(golden)} arrays, "
          f"{len(meta)} cases)")


if __name__ == "__main__":
    main(*sys.argv[1:])
