"""``LBMPipeNode``: MADDENING's pipe-flow node on the B200 kernels.

Drop-in for ``src/maddening/nodes/lbm_pipe.py:393-879``: D3Q19 fluid in a
cylindrical pipe along x, driven by an actuator-disc propeller (x body force
on one cross-section) and optional gravity (the value is added to the z force
of every fluid cell), periodic in x, bounce-back pipe walls.  Same constructor
arguments, validation, masks, state keys (``f``, ``density``, ``velocity``,
``tracer``, ``tracer_f``) and boundary input (``propeller_force``).

* ``G == 0`` (single phase): BGK with the Guo source, plus a D3Q7 passive
  tracer advected by the flow.
* ``G != 0`` (multiphase): Shan-Chen pseudopotential force with
  exact-difference forcing, a density floor, and the tracer read off the
  density (``tracer_f`` passes through).

The step runs in ``liblbm_b200.so`` (``lbm_pipe_rollout``); there is no CPU
path.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .contract import NodeMeta, SimulationNode, StabilityLevel, ValidatedRegime

_E = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
               [1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1],
               [1, 0, -1], [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]],
              dtype=np.int32)
_W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float32)
_W7 = np.array([1 / 4] + [1 / 8] * 6, dtype=np.float32)
_CS2 = 1.0 / 3.0


class lbm_pipe_args(C.Structure):
    _fields_ = [("wall", C.c_void_p), ("propeller", C.c_void_p), ("propeller_x", C.c_int32),
                ("propeller_force", C.c_double), ("gravity", C.c_double),
                ("tau_tracer", C.c_double), ("G", C.c_double), ("rho_liquid", C.c_double),
                ("rho_gas", C.c_double), ("rho_0", C.c_double), ("rho_wall", C.c_double)]


def _lib_pipe():
    h = _lib.lib()
    if not getattr(h, "_pipe_sigs", False):
        P = C.c_void_p
        h.lbm_pipe_workspace_bytes.argtypes = [P, C.POINTER(C.c_size_t)]
        h.lbm_pipe_workspace_bytes.restype = C.c_int
        h.lbm_pipe_rollout.argtypes = [P, P, P, P, P, P, C.c_int64, C.POINTER(lbm_pipe_args),
                                       C.POINTER(_lib.lbm_moments), P, P, C.c_size_t]
        h.lbm_pipe_rollout.restype = C.c_int
        h._pipe_sigs = True
    return h


def _cross_section_radius(ny, nz):
    """Distance of every (y, z) cell from the pipe axis, in float32 like the
    reference's ``jnp.arange(..., float32)`` grids (lbm_pipe.py:583-588)."""
    y = np.arange(ny, dtype=np.float32)
    z = np.arange(nz, dtype=np.float32)
    yy, zz = np.meshgrid(y, z, indexing="ij")
    cy, cz = (ny - 1) / 2.0, (nz - 1) / 2.0
    return np.sqrt((yy - np.float32(cy)) ** 2 + (zz - np.float32(cz)) ** 2), yy, zz


def _equilibrium(density, velocity):
    """lbm_pipe.py:144-167 (float32, the initial state)."""
    e_dot_u = velocity @ _E.astype(np.float32).T
    u_sq = np.sum(velocity ** 2, axis=-1, keepdims=True)
    return _W * density[..., None] * (1.0 + e_dot_u / _CS2 + e_dot_u ** 2 / (2.0 * _CS2 ** 2)
                                      - u_sq / (2.0 * _CS2))


def _tracer_equilibrium(tracer, velocity):
    """lbm_pipe.py:256-271."""
    return _W7 * tracer[..., None] * (1.0 + velocity @ _E[:7].astype(np.float32).T / _CS2)


class LBMPipeNode(SimulationNode):
    """3-D lattice-Boltzmann pipe with an actuator-disc propeller and a tracer."""

    meta = NodeMeta(
        algorithm_id="MADD-NODE-006",
        algorithm_version="1.0.0",
        stability=StabilityLevel.EXPERIMENTAL,
        description="D3Q19 Lattice Boltzmann in cylindrical pipe with propeller actuator disc "
                    "(B200 kernels)",
        governing_equations="BGK collision: f_i = f_i - (f_i - f_eq_i)/tau; "
                            "streaming: f_i(x+e_i, t+1) = f_i(x, t)",
        discretization="Lattice Boltzmann (D3Q19, explicit, 2nd-order in space and time for "
                       "low Ma)",
        assumptions=("Incompressible flow (Mach number << 1)",
                     "BGK single-relaxation-time collision operator",
                     "Rigid, impermeable pipe walls (bounce-back)",
                     "Periodic boundary conditions in flow direction",
                     "Actuator disc model for propeller (body force, not geometry)"),
        limitations=("Compressibility errors at high Mach number (Ma > 0.1)",
                     "BGK is less stable than MRT for high Reynolds numbers",
                     "No turbulence model", "Wall bounce-back is 1st-order at curved boundaries"),
        validated_regimes=(ValidatedRegime("tau", 0.501, 2.0, notes="tau > 0.5 required"),),
        hazard_hints=("Behaviour uncharacterised at Re > 100; validated only for laminar flow",),
    )

    def __init__(self, name: str, timestep: float, nx: int = 64, ny: int = 32, nz: int = 32,
                 tau: float = 0.8, pipe_radius: float = 0.9, propeller_x: int = 10,
                 propeller_radius: float = 0.8, propeller_strength: float = 0.0005,
                 initial_velocity: float = 0.0, gravity: float = 0.0,
                 fill_fraction: float = 1.0, tau_tracer: float = 0.6, G: float = 0.0,
                 rho_liquid: float = 1.0, rho_gas: float = 0.25, rho_0: float = 1.0,
                 rho_wall=None, *, storage: str = "f32", device=None):
        # validation in the reference's order and words (lbm_pipe.py:513-536)
        if tau <= 0.5:
            raise ValueError(f"tau must be > 0.5 for stability (got {tau}). "
                             f"nu = (tau - 0.5) / 3 = {(tau - 0.5) / 3:.4f}")
        if tau_tracer <= 0.5:
            raise ValueError(f"tau_tracer must be > 0.5 for stability (got {tau_tracer}).")
        if not 0.0 < fill_fraction <= 1.0:
            raise ValueError(f"fill_fraction must be in (0, 1] (got {fill_fraction}).")
        if G != 0.0:
            if rho_liquid <= rho_gas:
                raise ValueError(f"rho_liquid must be > rho_gas (got {rho_liquid} <= {rho_gas}).")
            if rho_gas <= 0.0:
                raise ValueError(f"rho_gas must be > 0 (got {rho_gas}).")
            if rho_0 <= 0.0:
                raise ValueError(f"rho_0 must be > 0 (got {rho_0}).")
        if storage not in ("f32", "f64"):
            raise ValueError(f"storage must be 'f32' or 'f64' (got {storage!r})")
        if rho_wall is None:
            rho_wall = rho_liquid
        super().__init__(name, timestep, nx=nx, ny=ny, nz=nz, tau=tau, pipe_radius=pipe_radius,
                         propeller_x=propeller_x, propeller_radius=propeller_radius,
                         propeller_strength=propeller_strength,
                         initial_velocity=initial_velocity, gravity=gravity,
                         fill_fraction=fill_fraction, tau_tracer=tau_tracer, G=G,
                         rho_liquid=rho_liquid, rho_gas=rho_gas, rho_0=rho_0, rho_wall=rho_wall)
        self._nx, self._ny, self._nz = int(nx), int(ny), int(nz)
        self._tau, self._tau_tracer = float(tau), float(tau_tracer)
        self._gravity = float(gravity)
        self._fill_fraction = float(fill_fraction)
        self._G = float(G)
        self._rho_liquid, self._rho_gas = float(rho_liquid), float(rho_gas)
        self._rho_0, self._rho_wall = float(rho_0), float(rho_wall)
        self._storage = storage
        self._io_dtype = torch.float64 if storage == "f64" else torch.float32
        self._device = torch.device(device) if device is not None else None
        r, _, _ = _cross_section_radius(ny, nz)
        max_r = pipe_radius * min(ny, nz) / 2.0
        cross_wall = r >= np.float32(max_r)
        self._wall_np = np.broadcast_to(cross_wall[None], (nx, ny, nz)).copy()
        prop_r = propeller_radius * pipe_radius * min(ny, nz) / 2.0
        self._prop2d = (r < np.float32(prop_r)) if 0 <= propeller_x < nx else \
            np.zeros((ny, nz), dtype=bool)
        self._prop_x = int(propeller_x)
        self._plan = _lib.Plan(19, (nx, ny, nz), tau, storage)
        self._dev_cache = {}

    # -- properties / contract ---------------------------------------------
    @property
    def viscosity(self) -> float:
        """Kinematic viscosity in lattice units."""
        return (self.params["tau"] - 0.5) / 3.0

    @property
    def wall_mask(self) -> np.ndarray:
        return self._wall_np

    @property
    def propeller_mask(self) -> np.ndarray:
        mask = np.zeros((self._nx, self._ny, self._nz), dtype=bool)
        if 0 <= self._prop_x < self._nx:
            mask[self._prop_x] = self._prop2d
        return mask

    def halo_width(self) -> dict:
        """One ghost cell per side on each spatial axis (lbm_pipe.py:656-662)."""
        return {0: 1, 1: 1, 2: 1}

    def derivatives(self, state, boundary_inputs):
        raise NotImplementedError("LBMPipeNode uses a discrete lattice Boltzmann update")

    def _dev(self) -> torch.device:
        if not torch.cuda.is_available():
            raise RuntimeError("LBMPipeNode needs a CUDA device (sm_100a); there is no CPU path")
        if self._device is None:
            self._device = torch.device("cuda", torch.cuda.current_device())
        return self._device

    def _on(self, dev, key, arr):
        k = (str(dev), key)
        if k not in self._dev_cache:
            self._dev_cache[k] = torch.as_tensor(arr.astype(np.uint8), device=dev).contiguous()
        return self._dev_cache[k]

    def _fill_mask(self) -> np.ndarray:
        """lbm_pipe.py:608-648."""
        ny, nz = self._ny, self._nz
        pipe_radius = self.params["pipe_radius"]
        cy, cz = (ny - 1) / 2.0, (nz - 1) / 2.0
        max_r = pipe_radius * min(ny, nz) / 2.0
        y = np.arange(ny, dtype=np.float32)
        z = np.arange(nz, dtype=np.float32)
        yy, zz = np.meshgrid(y, z, indexing="ij")
        interior = ~self._wall_np[0]
        z_cutoff = float(np.percentile(zz[interior], self._fill_fraction * 100))
        r = np.sqrt((yy - cy) ** 2 + (zz - cz) ** 2)
        near = ((max_r - r) < 1.5) & (np.abs(zz - z_cutoff) < 2.0)
        liquid = (zz <= z_cutoff) & interior & ~near
        return np.broadcast_to(liquid[None], (self._nx, ny, nz))

    def _multiphase_density(self) -> np.ndarray:
        """lbm_pipe.py:677-711: liquid below the fill level, gas above, joined
        by a tanh profile 5 cells wide; rho_gas in the walls."""
        ny, nz = self._ny, self._nz
        y = np.arange(ny, dtype=np.float32)
        z = np.arange(nz, dtype=np.float32)
        _, zz = np.meshgrid(y, z, indexing="ij")
        interior = ~self._wall_np[0]
        if self._fill_fraction >= 1.0:
            z_cutoff = float(nz)
        else:
            z_cutoff = float(np.percentile(zz[interior], self._fill_fraction * 100))
        phase = 0.5 * (1.0 + np.tanh((z_cutoff - np.arange(nz, dtype=np.float32)) / 5.0))
        phase_3d = np.broadcast_to(phase[None, None, :], (self._nx, ny, nz))
        density = self._rho_gas + (self._rho_liquid - self._rho_gas) * phase_3d
        return np.where(self._wall_np, self._rho_gas, density).astype(np.float32)

    def initial_state(self) -> dict:
        """lbm_pipe.py:664-749: uniform x velocity in the pipe, f = f_eq.
        Single phase: rho = 1, tracer = 1 in the (filled part of the) pipe.
        Multiphase: the tanh density profile, tracer read off the density."""
        dev = self._dev()
        fluid = ~self._wall_np
        shape = (self._nx, self._ny, self._nz)
        velocity = np.zeros(shape + (3,), dtype=np.float32)
        velocity[..., 0] = np.where(fluid, np.float32(self.params["initial_velocity"]),
                                    np.float32(0.0))
        if self._G != 0.0:
            density = self._multiphase_density()
            tracer = np.clip((density - self._rho_gas) / (self._rho_liquid - self._rho_gas),
                             0.0, 1.0)
            tracer = np.where(self._wall_np, 0.0, tracer).astype(np.float32)
        else:
            density = np.ones(shape, dtype=np.float32)
            liquid = fluid if self._fill_fraction >= 1.0 else self._fill_mask()
            tracer = np.where(liquid, 1.0, 0.0).astype(np.float32)
        f = _equilibrium(density, velocity).astype(np.float32)
        tracer_f = _tracer_equilibrium(tracer, velocity).astype(np.float32)
        to = lambda a: torch.as_tensor(a, device=dev).to(self._io_dtype)  # noqa: E731
        return {"f": to(f), "density": to(density), "velocity": to(velocity),
                "tracer": to(tracer), "tracer_f": to(tracer_f)}

    # -- stepping ------------------------------------------------------------
    def _advance(self, state: dict, boundary_inputs: dict, n_steps: int) -> dict:
        dev = self._dev()
        shape = (self._nx, self._ny, self._nz)

        def field(key, tail):
            t = torch.as_tensor(state[key], device=dev).to(self._io_dtype).contiguous()
            if tuple(t.shape) != shape + tail:
                raise ValueError(f"state[{key!r}] shape {tuple(t.shape)} != {shape + tail}")
            return t

        f = field("f", (19,))
        g = field("tracer_f", (7,))
        bi = boundary_inputs or {}
        s = bi.get("propeller_force", self.params["propeller_strength"])
        if isinstance(s, torch.Tensor):
            s = float(s.item())
        a = lbm_pipe_args()
        wall = self._on(dev, "wall", self._wall_np)
        prop = self._on(dev, "prop", self._prop2d)
        a.wall = wall.data_ptr()
        has_prop = 0 <= self._prop_x < self._nx
        a.propeller = prop.data_ptr() if has_prop else None
        a.propeller_x = self._prop_x if has_prop else 0
        a.propeller_force = float(s)
        a.gravity = self._gravity
        a.tau_tracer = self._tau_tracer
        a.G = self._G
        a.rho_liquid, a.rho_gas = self._rho_liquid, self._rho_gas
        a.rho_0, a.rho_wall = self._rho_0, self._rho_wall
        f_out = torch.empty_like(f)
        g_out = torch.empty_like(g)
        rho = torch.empty(shape, dtype=self._io_dtype, device=dev)
        vel = torch.empty(shape + (3,), dtype=self._io_dtype, device=dev)
        tracer = torch.empty(shape, dtype=self._io_dtype, device=dev)
        m = _lib.lbm_moments()
        m.density, m.velocity = rho.data_ptr(), vel.data_ptr()
        lib = _lib_pipe()
        nb = C.c_size_t()
        _lib.check(lib.lbm_pipe_workspace_bytes(self._plan.handle, C.byref(nb)))
        ws = torch.empty(int(nb.value), dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.lbm_pipe_rollout(self._plan.handle, stream, f.data_ptr(), f_out.data_ptr(),
                                        g.data_ptr(), g_out.data_ptr(), int(n_steps), C.byref(a),
                                        C.byref(m), tracer.data_ptr(), ws.data_ptr(), ws.numel()))
        return {"f": f_out, "density": rho, "velocity": vel, "tracer": tracer,
                "tracer_f": g_out}

    def update(self, state: dict, boundary_inputs: dict, dt: float) -> dict:
        """One step of lbm_pipe.py:751-879."""
        return self._advance(state, boundary_inputs, 1)

    def run(self, state: dict, boundary_inputs: dict, n_steps: int) -> dict:
        """``n_steps`` steps in one call (populations stay on the device)."""
        if int(n_steps) < 1:
            raise ValueError("n_steps must be >= 1")
        return self._advance(state, boundary_inputs, int(n_steps))
