"""CPU oracle for MADDENING's ``LBMPipeNode`` -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import it; the shipped path (``maddening_b200.pipe``) never
calls it.  A NumPy restatement of ``src/maddening/nodes/lbm_pipe.py`` that
follows the reference's operation order (single-phase mode, ``G == 0``):

* lattice constants (float32 weights, as the reference's ``_W``/``_W7``) --
  ``lbm_pipe.py:68-137``
* ``equilibrium`` / ``macroscopic`` (no half-force correction) /
  ``stream`` / ``guo_forcing``                     -- ``lbm_pipe.py:144-253``
* D3Q7 tracer ``tracer_equilibrium`` / ``stream7`` -- ``lbm_pipe.py:256-298``
* wall and propeller masks, fill mask            -- ``lbm_pipe.py:580-648``
* ``initial_state`` (single phase)               -- ``lbm_pipe.py:664-749``
* ``update``: collide with the raw velocity and the Guo source of the
  propeller + gravity force, periodic stream, wall-node swap, raw moments,
  u = 0 in walls; then the tracer: collide with the NEW velocity except in
  walls, stream, wall swap, tracer = sum (0 in walls)  -- ``lbm_pipe.py:751-879``

Multiphase mode (``G != 0``), same file:

* ``_psi`` / ``_shan_chen_force`` (Yuan-Schaefer pseudopotential, wall cells
  at psi(rho_wall), force zero in walls)        -- ``lbm_pipe.py:301-375``
* ``initial_state``: tanh density profile about the fill level, tracer from
  the density                                    -- ``lbm_pipe.py:677-726``
* ``update``: exact-difference forcing with the shifted velocity clamped to
  |u| <= 0.25, density floor 0.01 after the stream (populations rescaled),
  tracer from the new density, ``tracer_f`` passed through
                                                 -- ``lbm_pipe.py:775-864``

Modes: ``"x64"`` (FP64 arithmetic with the reference's float32 constants, as
under ``jax_enable_x64``) and ``"f32"``.  ``weights="exact"`` (x64 only)
replaces the reference's float32 lattice weights, which sum to 1 + 1.49e-8,
by 1/3, 1/18, 1/36: it isolates that rounding from the rest of the
arithmetic when an FP64 kernel is checked.
"""

from __future__ import annotations

import numpy as np

E = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
              [1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
              [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]], dtype=np.int32)
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float32)
W_EXACT = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float64)
OPP = np.array([0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15], dtype=np.int32)
CS2 = 1.0 / 3.0
E7 = E[:7].copy()
W7 = np.array([1 / 4] + [1 / 8] * 6, dtype=np.float32)
OPP7 = np.array([0, 2, 1, 4, 3, 6, 5], dtype=np.int32)


def _f(x, mode):
    return np.asarray(x, dtype=np.float64 if mode == "x64" else np.float32)


# Python-float constants, like the reference's: NumPy treats them as weak
# scalars (float32 arithmetic on float32 arrays), as JAX does.

def equilibrium(density, velocity, w=W):
    """lbm_pipe.py:144-167."""
    e_dot_u = velocity @ E.astype(np.float32).T
    u_sq = np.sum(velocity ** 2, axis=-1, keepdims=True)
    return w * density[..., None] * (1.0 + e_dot_u / CS2 + e_dot_u ** 2 / (2.0 * CS2 ** 2)
                                     - u_sq / (2.0 * CS2))


def macroscopic(f):
    """lbm_pipe.py:170-187 (no force correction)."""
    density = np.sum(f, axis=-1)
    momentum = f @ E.astype(np.float32)
    return density, momentum / np.maximum(density[..., None], 1e-10)


def stream(f, e):
    out = np.empty_like(f)
    for q in range(e.shape[0]):
        fq = f[..., q]
        for d in range(3):
            if e[q, d]:
                fq = np.roll(fq, int(e[q, d]), axis=d)
        out[..., q] = fq
    return out


def guo_forcing(density, velocity, force, tau, w=W):
    """lbm_pipe.py:218-253."""
    e_f = E.astype(np.float32)
    e_minus_u = e_f[None, None, None] - velocity[..., None, :]
    e_dot_u = velocity @ e_f.T
    e_scaled = e_f[None, None, None] * (e_dot_u / (CS2 ** 2))[..., None]
    bracket = e_minus_u / CS2 + e_scaled
    return (1.0 - 0.5 / tau) * w * np.sum(bracket * force[..., None, :], axis=-1)


def tracer_equilibrium(tracer, velocity):
    """lbm_pipe.py:256-271."""
    e_dot_u = velocity @ E7.astype(np.float32).T
    return W7 * tracer[..., None] * (1.0 + e_dot_u / CS2)


def psi(density, rho_0):
    """lbm_pipe.py:301-318."""
    return rho_0 * (1.0 - np.exp(-density / rho_0))


def shan_chen_force(density, G, rho_0, wall, rho_wall, w=W):
    """lbm_pipe.py:321-375: F(x) = -G psi(x) sum_q w_q psi(x + e_q) e_q, 0 in walls."""
    psi_wall = rho_0 * (1.0 - np.exp(-rho_wall / rho_0))
    psi_field = np.where(wall, psi_wall, psi(density, rho_0)).astype(density.dtype)
    e_f = E.astype(np.float32)
    grad = np.zeros(density.shape + (3,), dtype=np.float32)
    for q in range(19):
        w_q = float(w[q])
        shifted = psi_field
        for d in range(3):
            if E[q, d]:
                shifted = np.roll(shifted, -int(E[q, d]), axis=d)
        grad = grad + (w_q * shifted)[..., None] * e_f[q]
    force = -G * psi_field[..., None] * grad
    return np.where(wall[..., None], 0.0, force).astype(force.dtype)


def wall_mask(nx, ny, nz, pipe_radius):
    """lbm_pipe.py:580-592 (float32 coordinates, like jnp.arange(..., float32))."""
    y = np.arange(ny, dtype=np.float32)
    z = np.arange(nz, dtype=np.float32)
    yy, zz = np.meshgrid(y, z, indexing="ij")
    cy, cz = (ny - 1) / 2.0, (nz - 1) / 2.0
    r = np.sqrt((yy - np.float32(cy)) ** 2 + (zz - np.float32(cz)) ** 2)
    max_r = pipe_radius * min(ny, nz) / 2.0
    return np.broadcast_to((r >= np.float32(max_r))[None], (nx, ny, nz)).copy()


def propeller_mask(nx, ny, nz, prop_x, prop_radius, pipe_radius):
    """lbm_pipe.py:594-606."""
    y = np.arange(ny, dtype=np.float32)
    z = np.arange(nz, dtype=np.float32)
    yy, zz = np.meshgrid(y, z, indexing="ij")
    cy, cz = (ny - 1) / 2.0, (nz - 1) / 2.0
    r = np.sqrt((yy - np.float32(cy)) ** 2 + (zz - np.float32(cz)) ** 2)
    max_r = prop_radius * pipe_radius * min(ny, nz) / 2.0
    mask = np.zeros((nx, ny, nz), dtype=bool)
    mask[prop_x] = r < np.float32(max_r)
    return mask


class OraclePipe:
    """``LBMPipeNode``: single phase (``G == 0``) or Shan-Chen multiphase."""

    def __init__(self, nx=64, ny=32, nz=32, tau=0.8, pipe_radius=0.9, propeller_x=10,
                 propeller_radius=0.8, propeller_strength=0.0005, initial_velocity=0.0,
                 gravity=0.0, fill_fraction=1.0, tau_tracer=0.6, G=0.0, rho_liquid=1.0,
                 rho_gas=0.25, rho_0=1.0, rho_wall=None, mode="x64", weights="reference"):
        if tau <= 0.5 or tau_tracer <= 0.5:
            raise ValueError("tau and tau_tracer must be > 0.5")
        if weights not in ("reference", "exact") or (weights == "exact" and mode != "x64"):
            raise ValueError("weights: 'reference', or 'exact' in x64 mode")
        self.w = W if weights == "reference" else W_EXACT
        self.G, self.rho_liquid, self.rho_gas, self.rho_0 = G, rho_liquid, rho_gas, rho_0
        self.rho_wall = rho_liquid if rho_wall is None else rho_wall
        self.nx, self.ny, self.nz = nx, ny, nz
        self.tau, self.tau_tracer = tau, tau_tracer
        self.pipe_radius = pipe_radius
        self.prop_strength = propeller_strength
        self.u0 = initial_velocity
        self.gravity = gravity
        self.fill_fraction = fill_fraction
        self.mode = mode
        self.wall = wall_mask(nx, ny, nz, pipe_radius)
        self.prop = propeller_mask(nx, ny, nz, propeller_x, propeller_radius, pipe_radius)

    def fill_mask(self):
        """lbm_pipe.py:608-648."""
        ny, nz = self.ny, self.nz
        cy, cz = (ny - 1) / 2.0, (nz - 1) / 2.0
        max_r = self.pipe_radius * min(ny, nz) / 2.0
        y = np.arange(ny, dtype=np.float32)
        z = np.arange(nz, dtype=np.float32)
        yy, zz = np.meshgrid(y, z, indexing="ij")
        interior = ~self.wall[0]
        z_cutoff = float(np.percentile(zz[interior], self.fill_fraction * 100))
        r = np.sqrt((yy - cy) ** 2 + (zz - cz) ** 2)
        wall_dist = max_r - r
        near = (wall_dist < 1.5) & (np.abs(zz - z_cutoff) < 2.0)
        liquid = (zz <= z_cutoff) & interior & ~near
        return np.broadcast_to(liquid[None], (self.nx, ny, nz)).copy()

    def initial_state(self):
        """lbm_pipe.py:664-749 (float32 like the reference)."""
        fluid = ~self.wall
        shape = (self.nx, self.ny, self.nz)
        velocity = np.zeros(shape + (3,), dtype=np.float32)
        velocity[..., 0] = np.where(fluid, np.float32(self.u0), np.float32(0.0))
        if self.G != 0.0:
            return self._initial_state_multiphase(velocity)
        density = np.ones(shape, dtype=np.float32)
        f = equilibrium(density, velocity).astype(np.float32)
        if self.fill_fraction >= 1.0:
            tracer = np.where(fluid, 1.0, 0.0).astype(np.float32)
        else:
            tracer = np.where(self.fill_mask(), 1.0, 0.0).astype(np.float32)
        tracer_f = tracer_equilibrium(tracer, velocity).astype(np.float32)
        return {"f": f, "density": density, "velocity": velocity, "tracer": tracer,
                "tracer_f": tracer_f}

    def _initial_state_multiphase(self, velocity):
        """lbm_pipe.py:677-714: tanh density profile about the fill level."""
        ny, nz = self.ny, self.nz
        y = np.arange(ny, dtype=np.float32)
        z = np.arange(nz, dtype=np.float32)
        _, zz = np.meshgrid(y, z, indexing="ij")
        interior = ~self.wall[0]
        if self.fill_fraction >= 1.0:
            z_cutoff = float(nz)
        else:
            z_cutoff = float(np.percentile(zz[interior], self.fill_fraction * 100))
        z_dist = z_cutoff - np.arange(nz, dtype=np.float32)
        phase = 0.5 * (1.0 + np.tanh(z_dist / 5.0))
        phase_3d = np.broadcast_to(phase[None, None, :], (self.nx, ny, nz))
        density = self.rho_gas + (self.rho_liquid - self.rho_gas) * phase_3d
        density = np.where(self.wall, self.rho_gas, density).astype(np.float32)
        f = equilibrium(density, velocity).astype(np.float32)
        tracer = np.clip((density - self.rho_gas) / (self.rho_liquid - self.rho_gas), 0.0, 1.0)
        tracer = np.where(self.wall, 0.0, tracer).astype(np.float32)
        tracer_f = tracer_equilibrium(tracer, velocity).astype(np.float32)
        return {"f": f, "density": density, "velocity": velocity, "tracer": tracer,
                "tracer_f": tracer_f}

    def _forces(self, velocity, bi):
        """lbm_pipe.py:766-779: propeller x force on the disc, gravity on fluid."""
        s = bi.get("propeller_force", self.prop_strength)
        force = np.zeros_like(velocity)
        force[..., 0] = np.where(self.prop, s, 0.0)
        force[..., 2] = force[..., 2] + np.where(~self.wall, self.gravity, 0.0)
        return force

    def _update_multiphase(self, state, bi):
        """lbm_pipe.py:751-864 with G != 0."""
        f = _f(state["f"], self.mode)
        dt_ = f.dtype
        tau = self.tau
        density, velocity_raw = macroscopic(f)
        force = self._forces(velocity_raw, bi)
        sc = shan_chen_force(density, self.G, self.rho_0, self.wall, self.rho_wall, self.w)
        total = force + sc
        density_safe = np.maximum(density, 0.01)
        f_eq_bare = equilibrium(density, velocity_raw, self.w)
        u_shifted = velocity_raw + total / density_safe[..., None]
        u_mag = np.sqrt(np.sum(u_shifted ** 2, axis=-1, keepdims=True))
        scale = np.minimum(1.0, 0.25 / np.maximum(u_mag, 1e-10))
        u_shifted = u_shifted * scale
        f_eq_shifted = equilibrium(density, u_shifted, self.w)
        f_post = f - (f - f_eq_bare) / tau + (f_eq_shifted - f_eq_bare)
        f_str = stream(f_post, E)
        f_bc = np.where(self.wall[..., None], f_str[..., OPP], f_str)
        density_new, velocity_new = macroscopic(f_bc)
        rho_floor = 0.01
        ratio = np.maximum(density_new, rho_floor) / np.maximum(density_new, 1e-20)
        fix = density_new < rho_floor
        f_bc = np.where(fix[..., None], f_bc * ratio[..., None], f_bc).astype(dt_)
        density_new = np.where(fix, rho_floor, density_new).astype(dt_)
        velocity_new = np.where(self.wall[..., None], 0.0, velocity_new).astype(dt_)
        tracer = np.clip((density_new - self.rho_gas) / (self.rho_liquid - self.rho_gas),
                         0.0, 1.0)
        tracer = np.where(self.wall, 0.0, tracer).astype(dt_)
        return {"f": f_bc, "density": density_new, "velocity": velocity_new,
                "tracer": tracer, "tracer_f": np.asarray(state["tracer_f"])}

    def update(self, state, boundary_inputs=None, dt=1.0):
        """lbm_pipe.py:751-879."""
        bi = boundary_inputs or {}
        if self.G != 0.0:
            return self._update_multiphase(state, bi)
        mode = self.mode
        f = _f(state["f"], mode)
        density, velocity = macroscopic(f)
        force = self._forces(velocity, bi)
        f_eq = equilibrium(density, velocity, self.w)
        f_post = f - (f - f_eq) / self.tau
        f_post = f_post + guo_forcing(density, velocity, force, self.tau, self.w)
        f_str = stream(f_post, E)
        f_bc = np.where(self.wall[..., None], f_str[..., OPP], f_str)
        density_new, velocity_new = macroscopic(f_bc)
        velocity_new = np.where(self.wall[..., None], 0.0, velocity_new).astype(velocity_new.dtype)

        g = _f(state["tracer_f"], mode)
        tracer = np.sum(g, axis=-1)
        g_eq = tracer_equilibrium(tracer, velocity_new)
        g_post = np.where(self.wall[..., None], g, g - (g - g_eq) / self.tau_tracer)
        g_str = stream(g_post, E7)
        g_bc = np.where(self.wall[..., None], g_str[..., OPP7], g_str)
        tracer_new = np.where(self.wall, 0.0, np.sum(g_bc, axis=-1)).astype(g_bc.dtype)
        return {"f": f_bc, "density": density_new, "velocity": velocity_new,
                "tracer": tracer_new, "tracer_f": g_bc}

    def run(self, state, bi, n):
        for _ in range(n):
            state = self.update(state, bi)
        return state
