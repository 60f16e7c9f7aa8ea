"""Batched uneven ensembles: many independent lattices, one launch per step.

The reference batches only equal-shaped runs (``GraphManager.run_sweep`` =
``jax.vmap`` over ``lax.scan``, ``src/maddening/core/graph_manager.py:2807-2881``).
``LBMEnsemble`` advances lattices of different shapes, relaxation times,
forces, walls and faces together: every step is one persistent launch over a
tile list that covers all instances (``lbm_batch_rollout``), optionally
recorded once as a CUDA graph and replayed.  Each instance gives exactly what
its own ``LBMNode.run`` gives.

``autotune`` times the launch shapes (persistent grid size, tile order, graph
replay) on the actual ensemble and keeps the fastest; results are cached per
(lattice, storage, shapes, device) in memory and in a JSON file.
"""

from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .node import LBMNode


class lbm_batch_config(C.Structure):
    _fields_ = [("blocks_per_sm", C.c_int32), ("tile_order", C.c_int32),
                ("use_graph", C.c_int32), ("group_mib", C.c_int32)]


_SIGS = {
    "lbm_batch_create": ([C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)], C.c_int),
    "lbm_batch_destroy": ([C.c_void_p], C.c_int),
    "lbm_batch_workspace_bytes": ([C.c_void_p, C.POINTER(C.c_size_t)], C.c_int),
    "lbm_batch_rollout": ([C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                           C.c_int64, C.POINTER(_lib.lbm_step_args),
                           C.POINTER(_lib.lbm_moments), C.POINTER(lbm_batch_config),
                           C.c_void_p, C.c_size_t], C.c_int),
}


def _lib_batch():
    h = _lib.lib()
    if not getattr(h, "_batch_sigs", False):
        for name, (a, r) in _SIGS.items():
            getattr(h, name).argtypes = a
            getattr(h, name).restype = r
        h._batch_sigs = True
    return h


DEFAULT_CONFIG = {"blocks_per_sm": 0, "tile_order": 0, "use_graph": 1, "group_mib": 0}
_MEM_CACHE: dict = {}


def _cache_path() -> Path:
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return Path(base) / "maddening_b200" / "autotune.json"


class LBMEnsemble:
    """Independent ``LBMNode`` lattices advanced together on one GPU."""

    def __init__(self, nodes):
        nodes = list(nodes)
        if not nodes:
            raise ValueError("empty ensemble")
        q, sto = nodes[0]._Q, nodes[0].storage
        for n in nodes:
            if n._Q != q or n.storage != sto:
                raise ValueError("ensemble members must share lattice and storage")
        self.nodes = nodes
        self._plans = (C.c_void_p * len(nodes))(*[n.plan.handle.value for n in nodes])
        h = C.c_void_p()
        lib = _lib_batch()
        _lib.check(lib.lbm_batch_create(self._plans, len(nodes), C.byref(h)))
        self._h = h
        n_ = C.c_size_t()
        _lib.check(lib.lbm_batch_workspace_bytes(h, C.byref(n_)))
        self._ws_bytes = int(n_.value)
        self.config = dict(DEFAULT_CONFIG)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.lbm_batch_destroy(h)
            self._h = None

    @property
    def cells(self) -> int:
        return int(sum(np.prod(n._grid_shape) for n in self.nodes))

    def workspace_bytes(self) -> int:
        return self._ws_bytes

    def key(self) -> str:
        dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
        shapes = [n._grid_shape for n in self.nodes]
        raw = json.dumps([self.nodes[0]._Q, self.nodes[0].storage, shapes, dev])
        return hashlib.sha1(raw.encode()).hexdigest()

    def run(self, states, boundary_inputs, n_steps: int, config=None, workspace=None):
        """``n_steps`` steps of every member; returns one state dict per member."""
        if int(n_steps) < 1:
            raise ValueError("n_steps must be >= 1")
        n = len(self.nodes)
        if len(states) != n or len(boundary_inputs) != n:
            raise ValueError("one state and one boundary-input dict per member")
        dev = self.nodes[0]._dev()
        cfg = dict(self.config if config is None else config)
        args = (_lib.lbm_step_args * n)()
        moms = (_lib.lbm_moments * n)()
        f_in = (C.c_void_p * n)()
        f_out = (C.c_void_p * n)()
        keep, outs = [], []
        for i, (node, st, bi) in enumerate(zip(self.nodes, states, boundary_inputs)):
            fi = node._f_in(st, dev)
            a, k = node._step_args(st, bi or {}, dev)
            keep.append((fi, k))
            f, rho, vel, prs, m = node._outputs(dev)
            args[i] = a
            moms[i] = m
            f_in[i] = fi.data_ptr()
            f_out[i] = f.data_ptr()
            o = {"f": f, "density": rho, "velocity": vel, "pressure": prs}
            if "wall_mask" in st:
                o["wall_mask"] = st["wall_mask"]
            outs.append(o)
        ws = workspace
        if ws is None or ws.numel() < self._ws_bytes:
            ws = torch.empty(self._ws_bytes, dtype=torch.uint8, device=dev)
        c = lbm_batch_config(int(cfg["blocks_per_sm"]), int(cfg["tile_order"]),
                             int(cfg["use_graph"]), int(cfg.get("group_mib", 0)))
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib_batch().lbm_batch_rollout(self._h, stream, f_in, f_out, int(n_steps),
                                                  args, moms, C.byref(c), ws.data_ptr(),
                                                  ws.numel()))
        del keep
        return outs

    def autotune(self, states, boundary_inputs, n_steps: int = 20, candidates=None,
                 use_cache: bool = True):
        """Time the launch shapes on this ensemble; keep and return the fastest."""
        key = self.key()
        if use_cache:
            if key in _MEM_CACHE:
                self.config = dict(_MEM_CACHE[key]["config"])
                return self.config
            try:
                disk = json.loads(_cache_path().read_text())
                if key in disk:
                    self.config = dict(disk[key]["config"])
                    _MEM_CACHE[key] = disk[key]
                    return self.config
            except (OSError, ValueError):
                pass
        if candidates is None:
            candidates = [{"blocks_per_sm": b, "tile_order": o, "use_graph": g, "group_mib": 0}
                          for b in (0, 4, 8, 16) for o in (0, 1) for g in (0, 1)]
            candidates += [{"blocks_per_sm": b, "tile_order": 2, "use_graph": 1, "group_mib": m}
                           for b in (0, 8) for m in (48, 96)]
        dev = self.nodes[0]._dev()
        ws = torch.empty(self._ws_bytes, dtype=torch.uint8, device=dev)
        timings = []
        for cfg in candidates:
            self.run(states, boundary_inputs, 2, cfg, ws)  # warm-up (and graph path)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            self.run(states, boundary_inputs, n_steps, cfg, ws)
            e1.record()
            torch.cuda.synchronize()
            timings.append((e0.elapsed_time(e1), cfg))
        best_ms, best = min(timings, key=lambda t: t[0])
        self.config = dict(best)
        entry = {"config": best, "ms": best_ms, "steps": n_steps,
                 "timings": [[t, c] for t, c in timings]}
        _MEM_CACHE[key] = entry
        if use_cache:
            try:
                path = _cache_path()
                path.parent.mkdir(parents=True, exist_ok=True)
                disk = json.loads(path.read_text()) if path.exists() else {}
                disk[key] = entry
                path.write_text(json.dumps(disk))
            except (OSError, ValueError):
                pass
        return self.config


def uneven_ensemble(n: int = 64, seed: int = 0, lo: int = 32, hi: int = 160,
                    storage: str = "f32", device=None):
    """Seeded uneven D3Q19 ensemble: per-axis extents round(exp(U[ln lo, ln hi])),
    tau ~ U[0.55, 1.5], walls on the first and last z plane, periodic x/y,
    uniform body force (g_x, 0, 0) with g_x ~ U[1e-7, 1e-5].

    Returns (nodes, boundary_inputs)."""
    rng = np.random.default_rng(seed)
    nodes, bis = [], []
    for i in range(n):
        shape = tuple(int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))
                      for _ in range(3))
        tau = float(rng.uniform(0.55, 1.5))
        g = float(rng.uniform(1e-7, 1e-5))
        wall = np.zeros(shape, dtype=bool)
        wall[..., 0] = True
        wall[..., -1] = True
        nodes.append(LBMNode(f"m{i}", 1.0, grid_shape=shape, viscosity=(tau - 0.5) / 3.0,
                             wall_mask=wall, storage=storage, device=device))
        bis.append({"body_force": np.array([g, 0.0, 0.0], dtype=np.float32)})
    return nodes, bis
