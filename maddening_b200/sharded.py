"""Slab-sharded lattice-Boltzmann rollouts: one process per GPU.

The B200 counterpart of MADDENING's ``ShardedStencilNode`` around
``LBMNode.update_padded`` (``src/maddening/cloud/multigpu/sharded_node.py:116-
420``): each rank owns a slab of the global lattice along reference axis 0.

``ShardedLBM`` keeps its slab between steps in the kernels' own state layout
(post-collision normalised offsets, ``lbm_state_*`` of the C ABI), padded by
one slice on each side of axis 0 only.  A step pulls every population from
its upstream neighbour, so the first interior slice needs, from the previous
rank's last slice, only the populations whose axis-0 component is +1 (5 of
D3Q19, 3 of D2Q9), and the last interior slice the ones with -1 from the next
rank.  Per step each rank therefore

1. steps its two boundary slices (one ``lbm_state_step`` each),
2. sends their crossing populations to the neighbours and receives theirs
   into its pad slices (point-to-point, on a second stream with NCCL so that
   the transfer overlaps step 3; staged through host memory with gloo),
3. steps the interior slices, and waits for the exchange before the next step.

Bytes over the link per rank and step: 2 x 5 x n1 n2 populations in the
storage type (D3Q19 FP32 256 x 256: 2.6 MB), against 2 x 19 (n1 + 2)(n2 + 2)
for whole halo planes; HBM traffic per step: one state step of the slab
(152 B/cell FP32) instead of ``update_padded``'s three reference-layout
passes.  The results equal ``LBMNode.run`` on the whole lattice bit for bit
(16-bit storage included: each block seeds its stochastic rounding with the
whole lattice's cell index).  Axes 1 and 2 are not split and keep their
periodic wrap inside the kernels; pressure / velocity faces may sit on them,
not on the sharded axis 0.

``fill_halos`` refreshes a block padded on every axis in the reference layout,
for callers of ``LBMNode.update_padded`` (the reference's own sharded path).
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


def crossing_populations(lattice):
    """Indices of the populations whose reference-axis-0 component is +1 and
    -1: the ones that cross a slab face along axis 0 in a step."""
    e0 = np.asarray(lattice.e)[:, 0]
    return np.nonzero(e0 == 1)[0].tolist(), np.nonzero(e0 == -1)[0].tolist()


def exchange_slices(state: torch.Tensor, plus, minus, rank: int, world: int, group=None,
                    staged: bool = False) -> None:
    """Fill the pad slices of a slab state ``state`` (shape ``(Q, n + 2, slice)``,
    slices 1..n the interior) with the neighbours' crossing populations: pad
    slice 0 gets populations ``plus`` of the previous rank's last interior
    slice, pad slice n + 1 populations ``minus`` of the next rank's first one
    (periodic: rank 0's previous is the last rank).  Every rank of ``group``
    calls it with the same shapes, in the same step; ``staged``: move the
    messages through host memory (gloo)."""
    n = state.shape[1] - 2
    ip = torch.as_tensor(plus, device=state.device)
    im = torch.as_tensor(minus, device=state.device)
    send_next = state[ip, n]  # gathered copies, contiguous
    send_prev = state[im, 1]
    if world == 1:
        state[ip, 0] = send_next
        state[im, n + 1] = send_prev
        return
    if staged:
        send_next, send_prev = send_next.cpu(), send_prev.cpu()
    recv_prev = torch.empty_like(send_next)
    recv_next = torch.empty_like(send_prev)
    prev, nxt = (rank - 1) % world, (rank + 1) % world
    gprev = dist.get_global_rank(group, prev) if group is not None else prev
    gnext = dist.get_global_rank(group, nxt) if group is not None else nxt
    # Point-to-point messages between two ranks match in issue order, so with
    # two ranks (prev == next) the plus populations land in the plus buffer.
    ops = [dist.P2POp(dist.isend, send_next, gnext, group),
           dist.P2POp(dist.irecv, recv_prev, gprev, group),
           dist.P2POp(dist.isend, send_prev, gprev, group),
           dist.P2POp(dist.irecv, recv_next, gnext, group)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    state[ip, 0] = recv_prev.to(state.device)
    state[im, n + 1] = recv_next.to(state.device)


class ShardedLBM:
    """The rollout of a global ``LBMNode`` split into slabs along axis 0.

    ``node``: the global node (grid, walls, viscosity, lattice, storage, faces
    on axes 1 / 2 only).  Rank ``r`` of ``world`` owns slices
    ``[r n0 / world, (r + 1) n0 / world)``; ``n0`` must divide evenly.
    ``scatter`` loads a global state (every rank passes the same one), ``run``
    advances ``n`` steps, ``local_state`` is this rank's interior, ``gather``
    collects the global state on every rank."""

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
        self.pshape = (self.n0 + 2,) + tuple(grid[1:])
        self.slice = int(np.prod(grid[1:]))
        self._rows = np.arange(self.lo - 1, self.lo + self.n0 + 1) % grid[0]
        self._wall_pad = np.take(node._wall_np, self._rows, axis=0)
        self._plus, self._minus = crossing_populations(node.lattice)
        self._staged = dist.is_initialized() and dist.get_backend(group) == "gloo"
        self._state = None
        self._comm = None

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

    def _dev(self):
        return self.node._dev()

    def _block(self, arr, dev, dtype=None):
        """The padded slab (axis-0 rows lo - 1 .. lo + n0, periodic) of a
        global array."""
        t = torch.as_tensor(arr, device=dev)
        rows = torch.as_tensor(self._rows, device=dev)
        t = t.index_select(0, rows)
        return (t.to(dtype) if dtype is not None else t).contiguous()

    def _block_inputs(self, bi, dev):
        out = dict(bi)
        D = len(self.grid)
        f = bi.get("body_force", None)
        if f is not None and np.ndim(f) == D + 1:
            out["body_force"] = self._block(f, dev, self.node._io_dtype)
        if "wall_mask_update" in bi:
            out["wall_mask_update"] = self._block(bi["wall_mask_update"], dev)
        return out

    def _view(self, t):
        return t.view(self.node._Q, self.n0 + 2, self.slice)

    def _offset(self):
        # the whole lattice's index of the block's first cell, modulo 2^32
        return ((self.lo - 1) * self.slice) % (1 << 32)

    # -- state ---------------------------------------------------------------
    def scatter(self, state: dict) -> None:
        """Load this rank's slab of a global state (``f`` of shape (*grid, Q))."""
        node, dev = self.node, self._dev()
        # the first collide takes the first run's boundary inputs (the force),
        # as a rollout's does: it runs there
        self._f_pad = self._block(state["f"], dev, node._io_dtype)
        plan = node._padded_plan(self.pshape)
        nbytes = plan.state_bytes()
        self._bufs = [torch.empty(nbytes, dtype=torch.uint8, device=dev) for _ in range(2)]
        self._cur = 0
        self._k = 0  # steps done; after k >= 1 steps the held state pulls into step k
        self._wall = torch.as_tensor(self._wall_pad.astype(np.uint8), device=dev).contiguous()
        self._last_bi = {}
        self._state = True

    def _typed(self, buf):
        dt = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16,
              "f64": torch.float64}[self.node.storage]
        return self._view(buf.view(dt))

    def _exchange(self, buf):
        exchange_slices(self._typed(buf), self._plus, self._minus, self.rank, self.world,
                        self.group, self._staged)

    def local_state(self) -> dict:
        """This rank's interior: ``f``, ``density``, ``velocity``, ``pressure``
        after the steps run so far (the moments of the last step; zero before
        the first)."""
        if self._state is None:
            raise RuntimeError("scatter a state first")
        node, dev = self.node, self._dev()
        D = len(self.grid)
        if self._k == 0:
            z = torch.zeros(self.pshape[1:], dtype=node._io_dtype, device=dev)
            zeros = z.expand((self.n0,) + z.shape).contiguous()
            return {"f": self._f_pad[1:-1].clone(), "density": zeros.clone(),
                    "velocity": torch.zeros((self.n0,) + self.pshape[1:] + (D,),
                                            dtype=node._io_dtype, device=dev),
                    "pressure": zeros}
        plan = node._padded_plan(self.pshape)
        f = torch.empty(self.pshape + (node._Q,), dtype=node._io_dtype, device=dev)
        rho = torch.empty(self.pshape, dtype=node._io_dtype, device=dev)
        vel = torch.empty(self.pshape + (D,), dtype=node._io_dtype, device=dev)
        prs = torch.empty(self.pshape, dtype=node._io_dtype, device=dev)
        m = _lib.lbm_moments()
        m.density, m.velocity, m.pressure = rho.data_ptr(), vel.data_ptr(), prs.data_ptr()
        args, keep = node._step_args({"wall_mask": self._wall}, self._last_bi, dev,
                                     shape=self.pshape)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().lbm_state_to_f(plan.handle, stream,
                                             self._bufs[self._cur].data_ptr(), f.data_ptr(),
                                             C.byref(args), C.byref(m)))
        del keep
        return {"f": f[1:-1], "density": rho[1:-1], "velocity": vel[1:-1],
                "pressure": prs[1:-1]}

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
    def run(self, boundary_inputs: dict, n_steps: int) -> None:
        """``n_steps`` steps with the same boundary inputs."""
        if self._state is None:
            raise RuntimeError("scatter a state first")
        node, dev = self.node, self._dev()
        bi = self._block_inputs(boundary_inputs or {}, dev)
        self._check_inputs(bi)
        n = int(n_steps)
        if n <= 0:
            return
        self._last_bi = bi
        plan = node._padded_plan(self.pshape)
        args, keep = node._step_args({"wall_mask": self._wall}, bi, dev, shape=self.pshape)
        lib = _lib.lib()
        main = torch.cuda.current_stream(dev)
        if self._k == 0:
            # the first collide (with this call's inputs); the first step's f is
            # the pull from it, so the state is held as is after one step
            _lib.check(lib.lbm_state_from_f(plan.handle, main.cuda_stream,
                                            self._f_pad.data_ptr(),
                                            self._bufs[self._cur].data_ptr(), C.byref(args),
                                            self._offset()))
            self._exchange(self._bufs[self._cur])
            self._f_pad = None
            self._k, n = 1, n - 1
        overlap = self.world > 1 and not self._staged
        if overlap and self._comm is None:
            self._comm = torch.cuda.Stream(dev)
        off, n0 = self._offset(), self.n0

        def step(src, dst, first, count):
            _lib.check(lib.lbm_state_step(plan.handle, main.cuda_stream, src.data_ptr(),
                                          dst.data_ptr(), C.byref(args), first, count, off))

        for _ in range(n):
            src, dst = self._bufs[self._cur], self._bufs[1 - self._cur]
            if overlap and n0 > 2:
                step(src, dst, 1, 1)           # the boundary slices first
                step(src, dst, n0, 1)
                ev = torch.cuda.Event()
                ev.record(main)
                with torch.cuda.stream(self._comm):
                    self._comm.wait_event(ev)
                    self._exchange(dst)         # overlaps the interior step
                step(src, dst, 2, n0 - 2)
                main.wait_stream(self._comm)
            else:
                step(src, dst, 1, n0)
                self._exchange(dst)
            self._cur = 1 - self._cur
            self._k += 1
        del keep


__all__ = ["ShardedLBM", "crossing_populations", "exchange_slices", "fill_halos"]
