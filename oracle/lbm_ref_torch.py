"""Differentiable torch restatement of the reference step -- TEST INFRASTRUCTURE ONLY.

The same operations as ``oracle/lbm_ref.py`` (and the reference's
``src/maddening/nodes/lbm.py:180-353, 899-986``: moments with F/2, BGK + Guo
collide, periodic roll-stream, wall-node swap, output moments with u = 0 in
walls), written with torch ops so that ``torch.autograd`` differentiates it.
It stands in for ``jax.grad`` of the reference node (JAX is not installed) when
the hand-written adjoint is checked.  Face conditions are not included (the
differentiated rollout does not support them).  Only tests import it.
"""

from __future__ import annotations

import torch

from oracle.lbm_ref import Lattice


def _consts(lat: Lattice, ref: torch.Tensor):
    e = torch.as_tensor(lat.e, dtype=ref.dtype, device=ref.device)
    w = torch.as_tensor(lat.w, dtype=ref.dtype, device=ref.device)
    return e, w


def equilibrium(density, velocity, lat: Lattice):
    """lbm.py:180-206."""
    e, w = _consts(lat, velocity)
    cs2 = lat.cs2
    eu = velocity @ e.T
    usq = (velocity ** 2).sum(-1, keepdim=True)
    return w * density[..., None] * (1.0 + eu / cs2 + eu ** 2 / (2.0 * cs2 ** 2)
                                     - usq / (2.0 * cs2))


def macroscopic(f, lat: Lattice, force):
    """lbm.py:209-239."""
    e, _ = _consts(lat, f)
    density = f.sum(-1)
    momentum = f @ e + 0.5 * force
    return density, momentum / torch.clamp(density[..., None], min=1e-10)


def guo_forcing(density, velocity, force, tau, lat: Lattice):
    """lbm.py:307-353."""
    e, w = _consts(lat, velocity)
    cs2 = lat.cs2
    eu = velocity @ e.T
    bracket = (e - velocity[..., None, :]) / cs2 + e * (eu / cs2 ** 2)[..., None]
    return (1.0 - 0.5 / tau) * w * (bracket * force[..., None, :]).sum(-1)


def stream(f, lat: Lattice):
    """lbm.py:242-267."""
    out = []
    for q in range(lat.Q):
        fq = f[..., q]
        for d in range(lat.D):
            s = int(lat.e[q, d])
            if s:
                fq = torch.roll(fq, s, dims=d)
        out.append(fq)
    return torch.stack(out, dim=-1)


def update(f, wall, force, tau, lat: Lattice):
    """One reference step without faces (lbm.py:899-986); wall: bool grid."""
    density, velocity = macroscopic(f, lat, force)
    feq = equilibrium(density, velocity, lat)
    f_post = f - (f - feq) / tau + guo_forcing(density, velocity, force, tau, lat)
    f_str = stream(f_post, lat)
    opp = torch.as_tensor(lat.opp, dtype=torch.long, device=f.device)
    return torch.where(wall[..., None], f_str[..., opp], f_str)


def rollout(f0, wall, force, tau, lat: Lattice, n_steps: int, checkpoint: bool = True):
    """n_steps steps; returns (f, density, velocity with u = 0 in walls)."""
    if force.ndim == 1:
        force = force.expand(tuple(f0.shape[:-1]) + (lat.D,))
    f = f0
    for _ in range(n_steps):
        if checkpoint and torch.is_grad_enabled():
            f = torch.utils.checkpoint.checkpoint(update, f, wall, force, tau, lat,
                                                  use_reentrant=False)
        else:
            f = update(f, wall, force, tau, lat)
    density, velocity = macroscopic(f, lat, force)
    velocity = torch.where(wall[..., None], torch.zeros_like(velocity), velocity)
    return f, density, velocity
