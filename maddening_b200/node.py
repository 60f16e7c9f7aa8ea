"""``LBMNode``: the reference's lattice-Boltzmann node on B200 kernels.

Drop-in for MADDENING's ``LBMNode`` (``src/maddening/nodes/lbm.py:531-1036``):
same constructor arguments, validation messages, state keys and dtypes,
boundary inputs and ``update`` semantics.  The arithmetic runs in the sm_100a
kernels of ``liblbm_b200.so`` through its C ABI; state arrays are torch CUDA
tensors (the caching allocator owns them).  There is no CPU path: without a
CUDA device or without the built library the calls raise.

Additions beyond the reference (documented extensions):

* ``run(state, boundary_inputs, n_steps)`` -- ``n_steps`` reference steps in
  one call, populations kept on the device as offsets between steps.
* ``run_with_history(state, boundary_inputs, n_steps, every=, fields=)`` -- the
  same, also returning the stacked state after every ``every``-th step (the
  node's part of ``run_scan_with_history``).
* boundary input ``inlet_velocity`` (D,) -- velocity face at ``inlet_face``.
* ``outlet_condition="zero_gradient"`` -- zero-gradient face at
  ``outlet_face`` on every step.
* ``storage`` -- how populations are held between steps inside ``run``:
  ``"f32"`` (default), ``"f16"``/``"bf16"`` (normalised offsets, FP32
  arithmetic) or ``"f64"`` (FP64 throughout; state arrays are float64).
* ``cells_per_thread`` -- kernel form of the steps inside ``run``: ``None``
  (default: two neighbouring cells per thread for FP16/BF16 storage when the
  contiguous extent is even, else one), ``1`` or ``2`` (also for FP32).  Every
  form gives bit-identical results.
* ``one_pass`` -- ``update`` (and the first step of ``run``) reads the
  reference-layout ``f`` once in a tiled kernel (``None`` or ``True``, the
  default; FP32, FP16 and BF16 storage, last extent a multiple of 4) or runs
  as two passes (``False``); the results are bit-identical.
"""

from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib
from .contract import (BoundaryInputSpec, NodeMeta, SimulationNode, StabilityLevel,
                       ValidatedRegime)
from .lattice import by_name

_FACE_MAP = {"x_min": (0, "min"), "x_max": (0, "max"), "y_min": (1, "min"),
             "y_max": (1, "max"), "z_min": (2, "min"), "z_max": (2, "max")}


def prescribed_density(pressure, cs2: float = 1.0 / 3.0):
    """``pressure / cs2`` the way the reference evaluates it (lbm.py:956).

    cs2 is a weak Python scalar: a float32 input divides in float32, a
    float64 or Python input in float64.  Returns a Python float for host
    inputs and a 0-d CUDA tensor for device inputs.
    """
    if isinstance(pressure, torch.Tensor):
        if pressure.is_cuda:
            return pressure.reshape(()) / cs2
        pressure = pressure.numpy()
    p = np.asarray(pressure)
    if p.dtype == np.float32:
        return float(np.float32(p) / np.float32(cs2))
    return float(np.float64(p) / cs2)


class LBMNode(SimulationNode):
    """BGK lattice-Boltzmann node (D3Q19 / D2Q9) with wall-node bounce-back,
    Zou-He pressure faces and Guo body forcing, on sm_100a kernels."""

    meta = NodeMeta(
        algorithm_id="MADD-NODE-007",
        algorithm_version="1.0.0",
        stability=StabilityLevel.EXPERIMENTAL,
        description=("General LBM node with BGK collision, Zou-He pressure BCs, "
                     "and arbitrary wall-mask domains (B200 kernels)"),
        governing_equations=("BGK collision: f_i = f_i - (f_i - f_eq_i)/tau + S_guo; "
                             "streaming: f_i(x+e_i, t+1) = f_i(x, t)"),
        discretization="Lattice Boltzmann (D3Q19/D2Q9, explicit, 2nd-order)",
        assumptions=("Incompressible flow (Mach number << 1)",
                     "BGK single-relaxation-time collision operator",
                     "Rigid, impermeable walls (wall-node bounce-back)",
                     "Zou-He pressure boundary conditions at inlet/outlet"),
        limitations=("Compressibility errors at high Mach number (Ma > 0.1)",
                     "BGK is less stable than MRT for high Reynolds numbers",
                     "No turbulence model",
                     "Wall bounce-back is 1st-order at curved boundaries"),
        validated_regimes=(ValidatedRegime("tau", 0.501, 2.0,
                                           notes="tau > 0.5 required"),),
        hazard_hints=("Behaviour uncharacterised at Re > 100",
                      "Wall bounce-back assumes rigid, impermeable walls"),
    )

    def __init__(self, name: str, timestep: float, grid_shape: tuple = (64, 32, 32),
                 viscosity: float = 0.1, lattice: str = "D3Q19",
                 wall_mask: Optional[np.ndarray] = None, inlet_face: str = "x_min",
                 outlet_face: str = "x_max", geometry_source: Optional[str] = None,
                 *, outlet_condition: str = "pressure", storage: str = "f32",
                 device=None, cells_per_thread: Optional[int] = None,
                 one_pass: Optional[bool] = None):
        lat = by_name(lattice)
        if len(grid_shape) != lat.D:
            raise ValueError(f"grid_shape has {len(grid_shape)} dims but lattice "
                             f"{lat.name} requires {lat.D} dims.")
        tau = 0.5 + viscosity / lat.cs2
        if tau <= 0.5:
            raise ValueError(f"tau must be > 0.5 (got {tau}). Increase viscosity.")
        for face_name, face_label in (("inlet_face", inlet_face), ("outlet_face", outlet_face)):
            if face_label not in _FACE_MAP:
                raise ValueError(f"Unknown {face_name} '{face_label}'. "
                                 f"Supported: {list(_FACE_MAP.keys())}")
            axis, _ = _FACE_MAP[face_label]
            if axis >= lat.D:
                raise ValueError(f"{face_name} '{face_label}' uses axis {axis} but lattice "
                                 f"{lat.name} only has {lat.D} dimensions.")
        if outlet_condition not in ("pressure", "zero_gradient"):
            raise ValueError(f"Unknown outlet_condition '{outlet_condition}'. "
                             "Supported: ['pressure', 'zero_gradient']")
        if storage not in _lib.STORAGE:
            raise ValueError(f"Unknown storage '{storage}'. Supported: {list(_lib.STORAGE)}")
        super().__init__(name, timestep, grid_shape=grid_shape, viscosity=viscosity,
                         lattice=lattice, inlet_face=inlet_face, outlet_face=outlet_face,
                         geometry_source=geometry_source)
        self._lat = lat
        self._grid_shape = tuple(int(n) for n in grid_shape)
        self._D = lat.D
        self._Q = lat.Q
        self._tau = tau
        self._cs2 = lat.cs2
        self._inlet_face = inlet_face
        self._outlet_face = outlet_face
        self._outlet_condition = outlet_condition
        self._storage = storage
        self._io_dtype = torch.float64 if storage == "f64" else torch.float32
        self._device = torch.device(device) if device is not None else None
        if wall_mask is not None:
            wall_mask = np.asarray(wall_mask)
            if wall_mask.shape != self._grid_shape:
                raise ValueError(f"wall_mask shape {wall_mask.shape} != grid_shape "
                                 f"{self._grid_shape}")
            self._wall_np = wall_mask.astype(bool)
        else:
            self._wall_np = np.zeros(self._grid_shape, dtype=bool)
        self._has_walls = bool(self._wall_np.any())
        self._wall_dev = {}
        if cells_per_thread not in (None, 1, 2):
            raise ValueError(f"cells_per_thread must be None, 1 or 2 (got {cells_per_thread})")
        flags = 0
        if cells_per_thread == 1:
            flags |= _lib.PLAN_SINGLE_CELLS
        elif cells_per_thread == 2:
            flags |= _lib.PLAN_PAIRED_CELLS
        if one_pass is False:
            flags |= _lib.PLAN_TWO_PASS
        self._plan = _lib.Plan(lat.Q, self._grid_shape, tau, storage, flags)

    # -- properties (lbm.py:690-703) ---------------------------------------
    @property
    def tau(self) -> float:
        return self._tau

    @property
    def viscosity(self) -> float:
        return self._cs2 * (self._tau - 0.5)

    @property
    def lattice(self):
        return self._lat

    @property
    def storage(self) -> str:
        return self._storage

    @property
    def plan(self) -> _lib.Plan:
        return self._plan

    # -- contract ------------------------------------------------------------
    def halo_width(self) -> dict:
        """One ghost cell per side on every spatial axis (lbm.py:709-717)."""
        return {axis: 1 for axis in range(self._D)}

    @property
    def requires_halo(self) -> bool:
        """Pre-v0.3 spelling of ``bool(halo_width())``."""
        return bool(self.halo_width())

    def _dev(self) -> torch.device:
        if not torch.cuda.is_available():
            raise RuntimeError("LBMNode needs a CUDA device (sm_100a); there is no CPU path")
        if self._device is None:
            self._device = torch.device("cuda", torch.cuda.current_device())
        return self._device

    def _wall_mask_on(self, dev) -> torch.Tensor:
        key = str(dev)
        if key not in self._wall_dev:
            self._wall_dev[key] = torch.as_tensor(self._wall_np.astype(np.uint8), device=dev)
        return self._wall_dev[key]

    def initial_state(self) -> dict:
        """rho = 1, u = 0, f = f_eq, p = rho cs2, wall_mask uint8 (lbm.py:719-745)."""
        dev = self._dev()
        shape = self._grid_shape
        density = torch.ones(shape, dtype=self._io_dtype, device=dev)
        velocity = torch.zeros(shape + (self._D,), dtype=self._io_dtype, device=dev)
        f = self.equilibrium(None, None)
        pressure = density * self._cs2
        return {"f": f, "density": density, "velocity": velocity, "pressure": pressure,
                "wall_mask": self._wall_mask_on(dev).clone()}

    def equilibrium(self, density=None, velocity=None) -> torch.Tensor:
        """f_eq(rho, u) on the device (lbm.py:180-206); None means rho=1 / u=0."""
        dev = self._dev()
        f = torch.empty(self._grid_shape + (self._Q,), dtype=self._io_dtype, device=dev)
        rho = None if density is None else self._as_field(density, self._grid_shape, dev)
        u = None if velocity is None else self._as_field(velocity, self._grid_shape + (self._D,), dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().lbm_equilibrium(
            self._plan.handle, stream, None if rho is None else rho.data_ptr(),
            None if u is None else u.data_ptr(), f.data_ptr()))
        return f

    def _as_field(self, x, shape, dev) -> torch.Tensor:
        t = torch.as_tensor(x, device=dev).to(self._io_dtype)
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"expected shape {tuple(shape)}, got {tuple(t.shape)}")
        return t.contiguous()

    # -- boundary inputs (lbm.py:910-968) ------------------------------------
    def _step_args(self, state: dict, bi: dict, dev, shape=None, interior=None):
        """Builds the C step arguments; returns (args, keep-alive tensors).

        ``shape``: the lattice the arrays describe (default ``grid_shape``; the
        padded block for ``update_padded``).  ``interior``: for a padded block,
        its interior shape -- a body-force field of that shape is zero-padded
        by one cell per side (lbm.py:826-832)."""
        a = _lib.lbm_step_args()
        keep = []
        D = self._D
        shape = self._grid_shape if shape is None else tuple(shape)
        # wall mask precedence: wall_mask_update > state["wall_mask"] > node mask
        if "wall_mask_update" in bi:
            wall = torch.as_tensor(bi["wall_mask_update"], device=dev)
        elif "wall_mask" in state:
            wall = torch.as_tensor(state["wall_mask"], device=dev)
        else:
            wall = self._wall_mask_on(dev)
        if tuple(wall.shape) != shape:
            raise ValueError(f"wall mask shape {tuple(wall.shape)} != grid_shape {shape}")
        wall = (wall != 0).to(torch.uint8).contiguous() if wall.dtype != torch.uint8 \
            else wall.contiguous()
        keep.append(wall)
        a.wall = wall.data_ptr()

        dev_vals = [None] * 9  # inlet[3], outlet[3], force[3]
        use_dev = False

        force = bi.get("body_force", None)
        if force is None:
            a.force_mode = _lib.FORCE_NONE
        else:
            ft = force if isinstance(force, torch.Tensor) else torch.as_tensor(np.asarray(force))
            if ft.ndim == 1 and tuple(ft.shape) == (D,):
                a.force_mode = _lib.FORCE_UNIFORM
                if ft.is_cuda:
                    use_dev = True
                    for d in range(D):
                        dev_vals[6 + d] = ft[d].to(torch.float32)
                else:
                    vals = ft.to(torch.float32).numpy()  # the reference casts to float32
                    for d in range(D):
                        a.force[d] = float(vals[d])
                        dev_vals[6 + d] = float(vals[d])
            else:
                if interior is not None and tuple(ft.shape) == tuple(interior) + (D,):
                    ft = torch.nn.functional.pad(
                        torch.as_tensor(ft, device=dev).to(self._io_dtype).movedim(-1, 0),
                        (1, 1) * D).movedim(0, -1)
                field = self._as_field(ft, shape + (D,), dev)
                keep.append(field)
                a.force_mode = _lib.FORCE_FIELD
                a.force_field = field.data_ptr()

        p_in = bi.get("inlet_pressure", None)
        u_in = bi.get("inlet_velocity", None)
        p_out = bi.get("outlet_pressure", None)
        if p_in is not None and u_in is not None:
            raise ValueError("inlet_pressure and inlet_velocity are exclusive")

        def set_face(face: _lib.lbm_face_bc, slot: int, kind: int, label: str, value):
            nonlocal use_dev
            face.kind = kind
            face.face = _lib.FACES[label]
            if kind == _lib.BC_PRESSURE:
                rho = prescribed_density(value, self._cs2)
                if isinstance(rho, torch.Tensor):
                    use_dev = True
                    dev_vals[slot] = rho.to(torch.float32)
                else:
                    face.value[0] = rho
                    dev_vals[slot] = rho
            elif kind == _lib.BC_VELOCITY:
                ut = value if isinstance(value, torch.Tensor) else torch.as_tensor(np.asarray(value))
                if tuple(ut.shape) != (D,):
                    raise ValueError(f"inlet_velocity must have shape ({D},)")
                if ut.is_cuda:
                    use_dev = True
                    for d in range(D):
                        dev_vals[slot + d] = ut[d].to(torch.float32)
                else:
                    for d, v in enumerate(ut.to(torch.float64).numpy()):
                        face.value[d] = float(v)
                        dev_vals[slot + d] = float(v)

        if p_in is not None:
            set_face(a.inlet, 0, _lib.BC_PRESSURE, self._inlet_face, p_in)
        elif u_in is not None:
            set_face(a.inlet, 0, _lib.BC_VELOCITY, self._inlet_face, u_in)
        if self._outlet_condition == "zero_gradient":
            set_face(a.outlet, 3, _lib.BC_ZERO_GRADIENT, self._outlet_face, None)
        elif p_out is not None:
            set_face(a.outlet, 3, _lib.BC_PRESSURE, self._outlet_face, p_out)

        if use_dev:
            parts = [v if isinstance(v, torch.Tensor) else
                     torch.tensor(0.0 if v is None else v, dtype=torch.float32, device=dev)
                     for v in dev_vals]
            dv = torch.stack([p.reshape(()).to(device=dev, dtype=torch.float32) for p in parts])
            keep.append(dv)
            a.dev_values = dv.data_ptr()
        return a, keep

    def _outputs(self, dev):
        shape = self._grid_shape
        f = torch.empty(shape + (self._Q,), dtype=self._io_dtype, device=dev)
        rho = torch.empty(shape, dtype=self._io_dtype, device=dev)
        vel = torch.empty(shape + (self._D,), dtype=self._io_dtype, device=dev)
        prs = torch.empty(shape, dtype=self._io_dtype, device=dev)
        m = _lib.lbm_moments()
        m.density, m.velocity, m.pressure = rho.data_ptr(), vel.data_ptr(), prs.data_ptr()
        return f, rho, vel, prs, m

    def _f_in(self, state, dev) -> torch.Tensor:
        f = state["f"]
        f = torch.as_tensor(f, device=dev)
        if f.dtype != self._io_dtype:
            f = f.to(self._io_dtype)
        if tuple(f.shape) != self._grid_shape + (self._Q,):
            raise ValueError(f"state['f'] shape {tuple(f.shape)} != "
                             f"{self._grid_shape + (self._Q,)}")
        return f.contiguous()

    def _advance(self, state: dict, boundary_inputs: dict, n_steps: int) -> dict:
        dev = self._dev()
        f_in = self._f_in(state, dev)
        args, keep = self._step_args(state, boundary_inputs or {}, dev)
        f, rho, vel, prs, m = self._outputs(dev)
        nbytes = self._plan.workspace_bytes() if n_steps > 1 else self._plan.state_bytes()
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        lib = _lib.lib()
        if n_steps == 1:
            rc = lib.lbm_update(self._plan.handle, stream, f_in.data_ptr(), f.data_ptr(),
                                C.byref(args), C.byref(m), ws.data_ptr(), ws.numel())
        else:
            rc = lib.lbm_rollout(self._plan.handle, stream, f_in.data_ptr(), f.data_ptr(),
                                 int(n_steps), C.byref(args), C.byref(m), ws.data_ptr(),
                                 ws.numel())
        _lib.check(rc)
        del keep
        out = {"f": f, "density": rho, "velocity": vel, "pressure": prs}
        if "wall_mask" in state:
            out["wall_mask"] = state["wall_mask"]
        return out

    def run_with_history(self, state: dict, boundary_inputs: dict, n_steps: int, *,
                         every: int = 1,
                         fields=("f", "density", "velocity", "pressure")):
        """``n_steps`` fused steps that also return the state after every
        ``every``-th step -- the node's share of ``GraphManager.
        run_scan_with_history`` (graph_manager.py:2753-2805), which stacks the
        whole state after each step.  Returns ``(final_state, history)`` with
        ``history[key]`` of shape ``(n_steps // every, *field_shape)`` for each
        key of ``fields`` (``f`` is 76 bytes per cell and record: leave it out,
        or record sparsely, for long rollouts).  The records equal the outputs
        of ``run`` with that many steps, bit for bit."""
        n = int(n_steps)
        every = int(every)
        if n < 1 or every < 1:
            raise ValueError("n_steps and every must be >= 1")
        fields = tuple(fields)
        bad = set(fields) - {"f", "density", "velocity", "pressure"}
        if bad:
            raise ValueError(f"unknown history fields {sorted(bad)}")
        dev = self._dev()
        f_in = self._f_in(state, dev)
        args, keep = self._step_args(state, boundary_inputs or {}, dev)
        f, rho, vel, prs, m = self._outputs(dev)
        nrec = n // every
        shapes = {"f": self._grid_shape + (self._Q,), "density": self._grid_shape,
                  "velocity": self._grid_shape + (self._D,), "pressure": self._grid_shape}
        history = {k: torch.empty((nrec,) + shapes[k], dtype=self._io_dtype, device=dev)
                   for k in fields}
        h = _lib.lbm_history()
        for k, t in history.items():
            setattr(h, k, t.data_ptr() if nrec > 0 else None)
        ws = torch.empty(self._plan.workspace_bytes(), dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().lbm_rollout_history(
            self._plan.handle, stream, f_in.data_ptr(), f.data_ptr(), n, every, C.byref(args),
            C.byref(m), C.byref(h), ws.data_ptr(), ws.numel()))
        del keep
        out = {"f": f, "density": rho, "velocity": vel, "pressure": prs}
        if "wall_mask" in state:
            out["wall_mask"] = state["wall_mask"]
        return out, history

    def update(self, state: dict, boundary_inputs: dict, dt: float) -> dict:
        """One reference step (lbm.py:899-986)."""
        return self._advance(state, boundary_inputs, 1)

    def run(self, state: dict, boundary_inputs: dict, n_steps: int) -> dict:
        """``n_steps`` reference steps with the same boundary inputs, fused."""
        if int(n_steps) < 1:
            raise ValueError("n_steps must be >= 1")
        return self._advance(state, boundary_inputs, int(n_steps))

    def _padded_plan(self, pshape) -> _lib.Plan:
        plans = self.__dict__.setdefault("_padded_plans", {})
        if pshape not in plans:
            plans[pshape] = _lib.Plan(self._Q, pshape, self._tau, self._storage)
        return plans[pshape]

    def update_padded(self, state_padded, boundary_inputs, dt, *, static_padded=None,
                      shard_info=None):
        """Halo-aware step on a block padded by one cell per side of every
        spatial axis (lbm.py:747-897), as ``ShardedStencilNode`` calls it after
        a halo exchange: the whole block is collided, the interior streams
        across the halo, the wall swap and the faces act on the interior, and
        the outputs keep the input's halo entries.  ``state_padded`` holds
        ``f``, ``density``, ``velocity``, ``pressure`` (and ``wall_mask``) of
        the padded block; ``body_force`` may be (D,), a padded field or an
        interior-shaped field (zero-padded).  ``static_padded`` and
        ``shard_info`` are accepted for the contract and unused, as in the
        reference."""
        del static_padded, shard_info
        dev = self._dev()
        f = torch.as_tensor(state_padded["f"], device=dev).to(self._io_dtype).contiguous()
        D, Q = self._D, self._Q
        pshape = tuple(int(n) for n in f.shape[:-1])
        if len(pshape) != D or f.shape[-1] != Q:
            raise ValueError(f"state_padded['f'] must have shape (*padded_grid, {Q}) with "
                             f"{D} spatial axes; got {tuple(f.shape)}")
        if min(pshape) < 3:
            raise ValueError(f"padded extents {pshape}: one halo cell per side needs >= 3")
        interior = tuple(n - 2 for n in pshape)
        bi = boundary_inputs or {}
        if ("wall_mask_update" not in bi and "wall_mask" not in state_padded
                and pshape != self._grid_shape):
            raise ValueError("update_padded needs the padded wall mask: "
                             "state_padded['wall_mask'] or boundary_inputs['wall_mask_update']")
        plan = self._padded_plan(pshape)
        args, keep = self._step_args(state_padded, bi, dev, shape=pshape, interior=interior)

        def padded_field(key, shape):
            t = torch.as_tensor(state_padded[key], device=dev).to(self._io_dtype)
            if tuple(t.shape) != shape:
                raise ValueError(f"state_padded[{key!r}] shape {tuple(t.shape)} != {shape}")
            return t.clone().contiguous()

        rho = padded_field("density", pshape)
        vel = padded_field("velocity", pshape + (D,))
        prs = padded_field("pressure", pshape)
        f_out = torch.empty_like(f)
        m = _lib.lbm_moments()
        m.density, m.velocity, m.pressure = rho.data_ptr(), vel.data_ptr(), prs.data_ptr()
        ws = torch.empty(plan.state_bytes(), dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().lbm_update_padded(plan.handle, stream, f.data_ptr(),
                                                f_out.data_ptr(), C.byref(args), C.byref(m),
                                                ws.data_ptr(), ws.numel()))
        del keep
        out = {"f": f_out, "density": rho, "velocity": vel, "pressure": prs}
        if "wall_mask" in state_padded:
            out["wall_mask"] = state_padded["wall_mask"]
        return out

    def derivatives(self, state: dict, boundary_inputs: dict) -> dict:
        raise NotImplementedError(
            "LBMNode uses a discrete lattice Boltzmann update, "
            "not a continuous ODE. derivatives() is not applicable.")

    def compute_boundary_fluxes(self, state: dict, boundary_inputs: dict, dt: float) -> dict:
        """Mean pressure over the fluid cells of the outlet face (lbm.py:995-1017)."""
        pressure = torch.as_tensor(state["pressure"])
        axis, side = _FACE_MAP[self._outlet_face]
        idx = [slice(None)] * self._D
        idx[axis] = 0 if side == "min" else -1
        idx = tuple(idx)
        wall = torch.as_tensor(self._wall_np[idx], device=pressure.device)
        p_face = pressure[idx]
        fluid = (~wall).sum().to(pressure.dtype)
        p_sum = torch.where(wall, torch.zeros_like(p_face), p_face).sum()
        return {"outlet_pressure_avg": p_sum / torch.clamp(fluid, min=1.0)}

    def boundary_input_spec(self) -> dict:
        return {
            "inlet_pressure": BoundaryInputSpec(shape=(), description="Zou-He pressure at inlet face"),
            "outlet_pressure": BoundaryInputSpec(shape=(), description="Zou-He pressure at outlet face"),
            "inlet_velocity": BoundaryInputSpec(shape=(self._D,),
                                                description="Velocity at inlet face (extension)"),
            "body_force": BoundaryInputSpec(shape=(*self._grid_shape, self._D),
                                            coupling_type="additive",
                                            description="External body force field"),
            "wall_mask_update": BoundaryInputSpec(shape=self._grid_shape,
                                                  description="Runtime wall mask override (True=wall)"),
        }

    # -- differentiable rollout --------------------------------------------------
    def rollout(self, state: dict, boundary_inputs: dict, n_steps: int, *,
                checkpoint_every: int = 0) -> dict:
        """``n_steps`` fused steps, differentiable with respect to ``state["f"]``
        and ``boundary_inputs["body_force"]`` (field or (D,)) through the
        hand-written adjoint (``lbm_rollout_forward`` / ``lbm_rollout_backward``).

        Populations are checkpointed every ``checkpoint_every`` steps (0: the
        ceiling of sqrt(n_steps)); the backward recomputes each segment.  Walls
        and body forces only (no face conditions); FP32 or FP64 storage.
        """
        if int(n_steps) < 1:
            raise ValueError("n_steps must be >= 1")
        bi = dict(boundary_inputs or {})
        for key in ("inlet_pressure", "outlet_pressure", "inlet_velocity"):
            if key in bi:
                raise ValueError(f"rollout(): face condition '{key}' is not differentiable here")
        if self._outlet_condition != "pressure":
            raise ValueError("rollout(): the zero-gradient outlet is not differentiable here")
        dev = self._dev()
        f0 = torch.as_tensor(state["f"], device=dev)
        if f0.dtype != self._io_dtype:
            f0 = f0.to(self._io_dtype)
        force = bi.pop("body_force", None)
        if force is not None and not isinstance(force, torch.Tensor):
            force = torch.as_tensor(np.asarray(force, dtype=np.float32), device=dev)
        if force is not None:
            force = force.to(device=dev)
        wall_state = {k: v for k, v in state.items() if k == "wall_mask"}
        f, rho, vel, prs = _RolloutFn.apply(f0, force, self, wall_state, bi, int(n_steps),
                                            int(checkpoint_every))
        out = {"f": f, "density": rho, "velocity": vel, "pressure": prs}
        if "wall_mask" in state:
            out["wall_mask"] = state["wall_mask"]
        return out

    # -- diagnostics -----------------------------------------------------------
    def mass_momentum(self, f) -> torch.Tensor:
        """FP64 (sum rho, sum rho u) of a state f, reduced on the device."""
        dev = self._dev()
        f = self._f_in({"f": f}, dev)
        out = torch.empty(4, dtype=torch.float64, device=dev)
        ws = torch.empty(self._plan.reduce_workspace_bytes(), dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().lbm_mass_momentum(self._plan.handle, stream, f.data_ptr(),
                                                out.data_ptr(), ws.data_ptr(), ws.numel()))
        return out[: 1 + self._D]


class _RolloutFn(torch.autograd.Function):
    """Fused rollout whose backward is the checkpointed hand-written adjoint."""

    @staticmethod
    def forward(ctx, f0, force, node, wall_state, bi, n_steps, checkpoint_every):
        dev = f0.device
        plan = node.plan
        D, grid = node._D, node._grid_shape
        bi_full = dict(bi)
        keep = []
        if force is not None:
            if force.ndim == 1 and tuple(force.shape) == (D,):
                bi_full["body_force"] = force.detach().to(torch.float32).cpu().numpy()
            else:
                ff = node._as_field(force.detach(), grid + (D,), dev)
                keep.append(ff)
                bi_full["body_force"] = ff
        args, k2 = node._step_args(wall_state, bi_full, dev)
        keep.extend(k2)
        f_in = f0.detach().contiguous()
        f_out, rho, vel, prs, mom = node._outputs(dev)
        ws = torch.empty(plan.adjoint_workspace_bytes(n_steps, checkpoint_every),
                         dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().lbm_rollout_forward(
            plan.handle, stream, f_in.data_ptr(), f_out.data_ptr(), n_steps, checkpoint_every,
            C.byref(args), C.byref(mom), ws.data_ptr(), ws.numel()))
        ctx.node, ctx.args, ctx.keep, ctx.ws = node, args, keep, ws
        ctx.n_steps, ctx.K = n_steps, checkpoint_every
        ctx.force_shape = None if force is None else tuple(force.shape)
        ctx.force_dtype = None if force is None else force.dtype
        ctx.save_for_backward(f_in)
        return f_out, rho, vel, prs

    @staticmethod
    def backward(ctx, g_f, g_rho, g_vel, g_prs):
        (f_in,) = ctx.saved_tensors
        node = ctx.node
        dev = f_in.device
        io = node._io_dtype
        if g_prs is not None:  # pressure = density * cs2
            g_rho = g_prs * node._cs2 if g_rho is None else g_rho + g_prs * node._cs2

        def ptr(t):
            return None if t is None else t.to(io).contiguous().data_ptr()

        g_rho_c = None if g_rho is None else g_rho.to(io).contiguous()
        g_vel_c = None if g_vel is None else g_vel.to(io).contiguous()
        g_f_c = None if g_f is None else g_f.to(io).contiguous()
        want_force = ctx.force_shape is not None and ctx.needs_input_grad[1]
        want_f0 = ctx.needs_input_grad[0]
        gF = None
        if want_force:
            n = node._D if len(ctx.force_shape) == 1 else int(np.prod(ctx.force_shape))
            gF = torch.empty(n, dtype=torch.float64, device=dev)
        gf0 = torch.empty_like(f_in) if want_f0 else None
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().lbm_rollout_backward(
            node.plan.handle, stream, f_in.data_ptr(), ctx.n_steps, ctx.K, C.byref(ctx.args),
            None if g_rho_c is None else g_rho_c.data_ptr(),
            None if g_vel_c is None else g_vel_c.data_ptr(),
            None if g_f_c is None else g_f_c.data_ptr(),
            None if gF is None else gF.data_ptr(),
            None if gf0 is None else gf0.data_ptr(), ctx.ws.data_ptr(), ctx.ws.numel()))
        grad_force = None
        if gF is not None:
            grad_force = gF.reshape(ctx.force_shape).to(ctx.force_dtype)
        return gf0, grad_force, None, None, None, None, None
