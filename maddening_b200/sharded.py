"""Slab-sharded lattice-Boltzmann rollouts: one process per GPU.

The B200 counterpart of MADDENING's ``ShardedStencilNode`` around
``LBMNode.update_padded`` (``src/maddening/cloud/multigpu/sharded_node.py:116-
420``): each rank owns a slab of the global lattice along axis 0 and keeps it
permanently in a block padded by one halo cell per side of every spatial axis.
Before every step the halos are refreshed --

* axes 1 and 2 (not sharded): periodic copies inside the block;
* axis 0: the first and last interior planes go to the previous and next rank
  and come back as their halo planes, whole ``(n1 + 2) x (n2 + 2) x Q``
  planes that are contiguous in the ``(*grid, Q)`` layout, so the point-to-
  point send/receive (NCCL between GPUs, gloo on CPU) needs no packing --

then ``lbm_update_padded`` advances the interior (the whole block is
collided, the interior pulls across the halo, walls and faces act on the
interior).  Only halo planes cross between ranks; the periodic wrap of axis 0
joins the last rank to the first.  The lattice is periodic on every axis, as
the reference's stream is; pressure / velocity faces may sit on axes 1 and 2
(every slab spans them whole), not on the sharded axis 0.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch
import torch.distributed as dist

from . import _lib
from .node import _FACE_MAP, LBMNode


def _ring(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def fill_halos(fp: torch.Tensor, rank: int, world: int, group=None) -> None:
    """Refresh the halo cells of a padded D3Q19/D2Q9 block ``fp`` of shape
    ``(n0 + 2, n1 + 2[, n2 + 2], Q)`` in place: periodic copies along the
    unsharded axes, then the halo planes of axis 0 from the neighbouring ranks
    (a local periodic copy with one rank).  Every rank of ``group`` calls it
    with the same block shape, in the same step."""
    D = fp.dim() - 1
    inner = fp[1:-1]
    for ax in range(1, D):  # unsharded axes: periodic inside the block
        lo = [slice(None)] * (D + 1)
        hi = [slice(None)] * (D + 1)
        src_lo = [slice(None)] * (D + 1)
        src_hi = [slice(None)] * (D + 1)
        lo[ax], src_lo[ax] = 0, -2
        hi[ax], src_hi[ax] = -1, 1
        inner[tuple(lo)] = inner[tuple(src_lo)]
        inner[tuple(hi)] = inner[tuple(src_hi)]
    if world == 1:
        fp[0] = fp[-2]
        fp[-1] = fp[1]
        return
    prev, nxt = (rank - 1) % world, (rank + 1) % world
    gprev = dist.get_global_rank(group, prev) if group is not None else prev
    gnext = dist.get_global_rank(group, nxt) if group is not None else nxt
    # Order: to next, from prev, to prev, from next.  Point-to-point messages
    # between two ranks match in issue order, so with two ranks (prev == next)
    # the last plane of one rank lands in the other's left halo and the first
    # plane in its right halo.
    ops = [dist.P2POp(dist.isend, fp[-2], gnext, group),
           dist.P2POp(dist.irecv, fp[0], gprev, group),
           dist.P2POp(dist.isend, fp[1], gprev, group),
           dist.P2POp(dist.irecv, fp[-1], gnext, group)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()


class ShardedLBM:
    """The rollout of a global ``LBMNode`` split into slabs along axis 0.

    ``node``: the global node (grid, walls, viscosity, lattice, storage, faces
    on axes 1 / 2 only).  Rank ``r`` of ``world`` owns planes
    ``[r n0 / world, (r + 1) n0 / world)``; ``n0`` must divide evenly.
    ``scatter`` loads a global state (every rank passes the same one), ``run``
    advances ``n`` steps, ``local_state`` is this rank's interior, ``gather``
    collects the global state on every rank.  With gloo the padded blocks are
    staged through host memory for the exchange."""

    def __init__(self, node: LBMNode, group=None):
        self.node = node
        self.group = group
        self.rank, self.world = _ring(group)
        grid = tuple(node._grid_shape)
        if grid[0] % self.world:
            raise ValueError(f"axis 0 extent {grid[0]} does not divide among {self.world} ranks")
        if node._outlet_condition == "zero_gradient":
            self._check_face(node._outlet_face)
        self.grid = grid
        self.n0 = grid[0] // self.world
        self.lo = self.rank * self.n0
        self.pshape = (self.n0 + 2,) + tuple(n + 2 for n in grid[1:])
        # the padded wall mask of this slab: periodic wrap on every axis
        idx = np.arange(self.lo - 1, self.lo + self.n0 + 1) % grid[0]
        wall = np.take(node._wall_np, idx, axis=0)
        self._wall_pad = np.pad(wall, [(0, 0)] + [(1, 1)] * (len(grid) - 1), mode="wrap")
        self._staged = dist.is_initialized() and dist.get_backend(group) == "gloo"
        self._bufs = None

    @staticmethod
    def _check_face(face):
        if _FACE_MAP[face][0] == 0:
            raise ValueError(f"face {face!r} lies on the sharded axis 0: put the faces on "
                             "axis 1 or 2")

    def _check_inputs(self, bi):
        if "inlet_pressure" in bi or "inlet_velocity" in bi:
            self._check_face(self.node._inlet_face)
        if "outlet_pressure" in bi:
            self._check_face(self.node._outlet_face)

    # -- state ---------------------------------------------------------------
    def _dev(self):
        return self.node._dev()

    def scatter(self, state: dict) -> None:
        """Load this rank's slab of a global state (``f`` of shape (*grid, Q))."""
        dev = self._dev()
        f = torch.as_tensor(state["f"], device=dev).to(self.node._io_dtype)
        Q = f.shape[-1]
        fp = torch.zeros(self.pshape + (Q,), dtype=f.dtype, device=dev)
        fp[1:-1][(slice(None),) + (slice(1, -1),) * (len(self.grid) - 1)] = \
            f[self.lo: self.lo + self.n0]
        D = len(self.grid)
        self._bufs = {
            "f": [fp, torch.empty_like(fp)],
            "density": torch.zeros(self.pshape, dtype=f.dtype, device=dev),
            "velocity": torch.zeros(self.pshape + (D,), dtype=f.dtype, device=dev),
            "pressure": torch.zeros(self.pshape, dtype=f.dtype, device=dev),
            "wall": torch.as_tensor(self._wall_pad.astype(np.uint8), device=dev).contiguous(),
        }
        self._cur = 0

    def _interior(self, t):
        return t[1:-1][(slice(None),) + (slice(1, -1),) * (len(self.grid) - 1)]

    def local_state(self) -> dict:
        """This rank's interior: ``f``, ``density``, ``velocity``, ``pressure``."""
        b = self._bufs
        return {"f": self._interior(b["f"][self._cur]), "density": self._interior(b["density"]),
                "velocity": self._interior(b["velocity"]),
                "pressure": self._interior(b["pressure"])}

    def gather(self) -> dict:
        """The global state on every rank (slabs concatenated along axis 0)."""
        loc = {k: v.contiguous() for k, v in self.local_state().items()}
        if self.world == 1:
            return loc
        out = {}
        for k, v in loc.items():
            src = v.cpu() if self._staged else v
            parts = [torch.empty_like(src) for _ in range(self.world)]
            dist.all_gather(parts, src, group=self.group)
            out[k] = torch.cat(parts, dim=0).to(v.device)
        return out

    # -- stepping --------------------------------------------------------------
    def _exchange(self, fp):
        if not self._staged:
            fill_halos(fp, self.rank, self.world, self.group)
            return
        host = fp.cpu()
        fill_halos(host, self.rank, self.world, self.group)
        fp.copy_(host)

    def run(self, boundary_inputs: dict, n_steps: int) -> None:
        """``n_steps`` steps: halo refresh, then the padded step, each step."""
        if self._bufs is None:
            raise RuntimeError("scatter a state first")
        node, dev = self.node, self._dev()
        boundary_inputs = boundary_inputs or {}
        self._check_inputs(boundary_inputs)
        b = self._bufs
        interior = tuple(n - 2 for n in self.pshape)
        plan = node._padded_plan(self.pshape)
        ws = torch.empty(plan.state_bytes(), dtype=torch.uint8, device=dev)
        m = _lib.lbm_moments()
        m.density, m.velocity = b["density"].data_ptr(), b["velocity"].data_ptr()
        m.pressure = b["pressure"].data_ptr()
        lib = _lib.lib()
        stream = torch.cuda.current_stream(dev).cuda_stream
        for _ in range(int(n_steps)):
            src, dst = b["f"][self._cur], b["f"][1 - self._cur]
            self._exchange(src)
            state = {"f": src, "wall_mask": b["wall"]}
            args, keep = node._step_args(state, boundary_inputs, dev, shape=self.pshape,
                                         interior=interior)
            _lib.check(lib.lbm_update_padded(plan.handle, stream, src.data_ptr(), dst.data_ptr(),
                                             C.byref(args), C.byref(m), ws.data_ptr(),
                                             ws.numel()))
            del keep
            self._cur = 1 - self._cur


__all__ = ["ShardedLBM", "fill_halos"]
