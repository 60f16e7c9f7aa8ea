"""Benchmark of the lattice-Boltzmann node step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 256^3 D3Q19 obstacle flow -- seeded random spheres (radii 4-12,
10% solid, centres >= 16 cells from the x faces), velocity inlet u=(0.05,0,0)
at x_min, zero-gradient outlet at x_max, periodic y/z, tau = 0.6, f0 = f_eq(1,0).
A "step" is one lattice update of all 16.8 M cells; the metric is MLUPS
(cells x steps / s / 1e6, wall cells included, as the kernel updates them).

* ``value``: K steps of ``lbm_rollout`` on device-resident buffers, timed
  with CUDA events on the launching stream (state 2 x 1.27 GB > L2, so no
  flush is needed between steps).
* ``e2e``: the same K steps through the public ``LBMNode.run`` with the state
  in pinned host memory: host->device copy of f and the wall mask, the
  rollout, device->host copy of f, density, velocity and pressure, all inside
  the timed region (bytes reported per lattice step).
* ``roofline``: 152 algorithmic bytes per cell-update (19 loads + 19 stores of
  4 B) of the state-step kernel over its average launch time, measured with
  CUDA events as (t(K steps) - t(2 steps)) / (K - 2), against the measured
  HBM copy bandwidth.
* ``update_call``: one ``LBMNode.update`` per step (the call a graph manager
  makes), reference-layout state in and out of every call.
* ``clocks``: SM clock and throttle reasons sampled through NVML every 2 ms
  from the warm-up to the end of the timed region.
* ``cpu_baseline``: the CPU restatement of the reference step (the oracle) on
  a bounded sample of the same workload, one process per host core.
* ``--impl reference``: the reference's CPU implementation of the path.  JAX
  (the reference's array runtime) is not installed on this image, so the
  restatement of the reference step stands in for it, on all host cores.

Multi-GPU (torchrun, one process per GPU): independent replicas of the
workload, no collective on the data path ("scaling": "weak").
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import multiprocessing as mp
import os
import platform
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRID = (256, 256, 256)
TAU = 0.6
U_IN = (0.05, 0.0, 0.0)
BYTES_PER_CELL = 152  # D3Q19 FP32: 19 x 4 B read + 19 x 4 B written
# DRAM bytes of one state step launch (k_step<19, float>) of the 256^3 FP32
# workload, from one capture of
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum
#       --clock-control none -k regex:k_step -s 5 -c 3 python bench.py --steps 20 --warmup 3
#       --no-cpu-baseline --no-variants
# (one pass): 1.29 GB read + 1.22 GB written per launch, against 2.55 GB
# algorithmic (the remainder of the writes is still in L2 when the launch ends).
NCU_TRAFFIC_256_F32 = 2.51e9
METRIC = "MLUPS (D3Q19 FP32 lattice updates/s) & HBM roofline fraction"
# the state-step kernel each storage form runs on the workload (rows of 256 cells)
KERNEL_LABEL = {
    "f32": "k_step<19,float,kOutState,faces,no force> (fused pull-stream-collide, one cell "
           "per thread)",
    "f64": "k_step<19,double,kOutState,faces,no force> (one cell per thread)",
    "f16": "k_step_quad<19,__half,faces,no force,2> (four cells per thread, 64-bit words)",
    "bf16": "k_step_quad<19,__nv_bfloat16,faces,no force,2> (four cells per thread)",
}
WORKLOAD = "256^3 D3Q19 obstacle flow, velocity inlet + zero-gradient outlet, tau 0.6"


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU side (oracle restatement): bounded samples
# ---------------------------------------------------------------------------

def _cpu_sample_worker(args):
    """One process: float32 restatement of the reference step on a slab of the
    workload (its first ``nx`` x-planes, same boundary conditions)."""
    nx, steps, seed = args
    from oracle import lbm_ref as R
    from maddening_b200.geometry import random_spheres
    grid = (nx, GRID[1], GRID[2])
    wall = random_spheres(GRID, seed=seed)[:nx]
    node = R.OracleLBM(grid, (TAU - 0.5) / 3.0, "D3Q19", wall_mask=wall,
                       outlet_condition="zero_gradient", mode="f32")
    st = node.initial_state()
    st["f"] = st["f"].astype(np.float32)
    bi = {"inlet_velocity": np.array(U_IN)}
    st = node.update(st, bi)  # warm-up
    t0 = time.perf_counter()
    for _ in range(steps):
        st = node.update(st, bi)
    dt = time.perf_counter() - t0
    return nx * GRID[1] * GRID[2] * steps, dt


def cpu_baseline(procs: int, nx: int, steps: int):
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        t0 = time.perf_counter()
        res = pool.map(_cpu_sample_worker, [(nx, steps, 0)] * procs)
        wall_s = time.perf_counter() - t0
    cells = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    return cells / busy / 1e6, wall_s


def _host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:  # noqa: BLE001
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    """SM clock, power and throttle reasons of one GPU, read through NVML (read
    only) by a thread every ``period`` seconds while the context is open."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown",
               0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap"}

    def __init__(self, torch_device, period: float = 0.002):
        self.period = period
        self.rows = []
        self.err = None
        self._stop = threading.Event()
        self._thread = None
        self._h = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            self._nv = pynvml
            try:
                props = torch.cuda.get_device_properties(torch_device)
                bus = "%08x:%02x:%02x.0" % (props.pci_domain_id, props.pci_bus_id,
                                            props.pci_device_id)
                self._h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:  # noqa: BLE001
                self._h = pynvml.nvmlDeviceGetHandleByIndex(torch.device(torch_device).index or 0)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
        except Exception as e:  # noqa: BLE001
            self.err = f"NVML unavailable: {e}"

    def _sample(self):
        nv = self._nv
        try:
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        except AttributeError:
            reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self._h)
        self.rows.append((time.perf_counter(),
                          float(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)),
                          nv.nvmlDeviceGetPowerUsage(self._h) / 1000.0, int(reasons)))

    def _run(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception as e:  # noqa: BLE001
                self.err = str(e)
                return
            self._stop.wait(self.period)

    def __enter__(self):
        if self._h is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)

    def summary(self, t0=None, t1=None):
        """Median SM clock and the reasons seen; with t0/t1 (perf_counter
        seconds) also the samples taken inside that window."""
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.err or "no samples"]}
        sm = [r[1] for r in self.rows]
        loaded = [x for x in sm if x > 0.5 * max(sm)]
        reasons = sorted({name for r in self.rows for bit, name in self.REASONS.items()
                          if r[3] & bit})
        out = {"sm_mhz": statistics.median(loaded), "sm_max_mhz": self.max_mhz,
               "reasons": reasons, "samples": len(self.rows), "source": "NVML",
               "power_w_max": round(max(r[2] for r in self.rows), 1)}
        if t0 is not None:
            inside = [r[1] for r in self.rows if t0 <= r[0] <= t1]
            out["samples_in_timed_region"] = len(inside)
            if inside:
                out["sm_mhz_timed_region"] = statistics.median(inside)
        return out


def host_info():
    model = platform.processor() or "unknown"
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "cpu_count": os.cpu_count(), "affinity": _host_cores(),
            "reference_runtime": "reference JAX CPU path unavailable on this machine (jax is not "
                                 "installed and has no offline wheel); the float32 "
                                 "restatement of the reference step stands in"}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def _dist_init():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def _barrier(world):
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def _max_over_ranks(world, value):
    """The largest ``value`` of all ranks (device timings: the job's time)."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return value
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _job_mlups(world, cells, steps, t_max):
    """Whole-job throughput of ``world`` replicas of ``cells`` x ``steps``
    lattice updates, timed as the slowest rank's ``t_max`` seconds."""
    return world * cells * steps / t_max / 1e6


def run_ours(args):
    import torch
    from maddening_b200 import LBMNode, _lib
    from maddening_b200.geometry import random_spheres

    world, rank, local = _dist_init()
    dev = torch.device("cuda", local)
    cells = GRID[0] * GRID[1] * GRID[2]
    wall = random_spheres(GRID, seed=0)
    node = LBMNode("bench", 1.0, grid_shape=GRID, viscosity=(TAU - 0.5) / 3.0,
                   wall_mask=wall, outlet_condition="zero_gradient", device=dev,
                   storage=args.storage)
    io_dtype = torch.float64 if args.storage == "f64" else torch.float32
    bytes_per_cell = {"f32": 152, "f16": 76, "bf16": 76, "f64": 304}[args.storage]
    bi = {"inlet_velocity": np.array(U_IN)}

    # device-resident buffers for the kernel-throughput number
    st = node.initial_state()
    f_a = st["f"]
    f_b = torch.empty_like(f_a)
    plan = node.plan
    ws = torch.empty(plan.workspace_bytes(), dtype=torch.uint8, device=dev)
    sargs, keep = node._step_args(st, bi, dev)
    rho = torch.empty(GRID, device=dev, dtype=io_dtype)
    vel = torch.empty(GRID + (3,), device=dev, dtype=io_dtype)
    prs = torch.empty(GRID, device=dev, dtype=io_dtype)
    mom = _lib.lbm_moments()
    mom.density, mom.velocity, mom.pressure = rho.data_ptr(), vel.data_ptr(), prs.data_ptr()
    lib = _lib.lib()
    stream = torch.cuda.current_stream(dev)

    def rollout(src, dst, n):
        _lib.check(lib.lbm_rollout(plan.handle, stream.cuda_stream, src.data_ptr(),
                                   dst.data_ptr(), int(n), C.byref(sargs), C.byref(mom),
                                   ws.data_ptr(), ws.numel()))

    K = args.steps
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        rollout(f_a, f_b, max(args.warmup, 3))
        _barrier(world)
        w0 = time.perf_counter()
        e0.record(stream)
        rollout(f_b, f_a, K)
        e1.record(stream)
        _barrier(world)
        w1 = time.perf_counter()
    t_dev = e0.elapsed_time(e1) / 1e3
    t_dev = _max_over_ranks(world, t_dev)
    mlups = _job_mlups(world, cells, K, t_dev)
    clocks = clk.summary(w0, w1)
    if clocks.get("sm_mhz"):
        clocks["ms_x_median_sm_ghz"] = round(t_dev / K * 1e3 * clocks["sm_mhz"] / 1e3, 4)
    # the state-step kernel alone: a rollout of K steps is the first step, K - 2
    # state steps and the last step; one of 2 steps has the first and last only
    e4 = torch.cuda.Event(enable_timing=True)
    e5 = torch.cuda.Event(enable_timing=True)
    rollout(f_a, f_b, 2)
    e4.record(stream)
    for _ in range(5):
        rollout(f_a, f_b, 2)
    e5.record(stream)
    torch.cuda.synchronize()
    t_two = e4.elapsed_time(e5) / 5 / 1e3
    t_kernel = (t_dev - t_two) / (K - 2) if K > 2 else t_dev / K

    # e2e: public API, state in pinned host memory
    f_host = f_a.cpu().pin_memory()
    wall_host = torch.as_tensor(wall.astype(np.uint8)).pin_memory()
    outs = {k: torch.empty(s, dtype=io_dtype).pin_memory() for k, s in
            (("f", GRID + (19,)), ("density", GRID), ("velocity", GRID + (3,)),
             ("pressure", GRID))}
    state_host = {"f": f_host, "wall_mask": wall_host}

    def e2e_once(n):
        dstate = {"f": state_host["f"].to(dev, non_blocking=True),
                  "wall_mask": state_host["wall_mask"].to(dev, non_blocking=True)}
        res = node.run(dstate, bi, n)
        for k in outs:
            outs[k].copy_(res[k], non_blocking=True)

    e2e_once(3)
    _barrier(world)
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    e2e_once(K)
    e3.record(stream)
    _barrier(world)
    t_e2e = _max_over_ranks(world, e2.elapsed_time(e3) / 1e3)
    h2d = f_host.numel() * f_host.element_size() + wall_host.numel()
    d2h = sum(v.numel() * v.element_size() for v in outs.values())

    # variants: other storage forms of the same workload (informational)
    variants = {}
    if not args.no_variants:
        for storage in ("f16", "bf16"):
            vn = LBMNode("v", 1.0, grid_shape=GRID, viscosity=(TAU - 0.5) / 3.0,
                         wall_mask=wall, outlet_condition="zero_gradient", storage=storage,
                         device=dev)
            vs = vn.initial_state()
            vn.run(vs, bi, 3)
            torch.cuda.synchronize()

            def timed_run(n):
                a0 = torch.cuda.Event(enable_timing=True)
                a1 = torch.cuda.Event(enable_timing=True)
                a0.record(stream)
                vn.run(vs, bi, n)
                a1.record(stream)
                torch.cuda.synchronize()
                return a0.elapsed_time(a1) / 1e3

            tv = timed_run(K)
            t2 = min(timed_run(2) for _ in range(3))
            tk = (tv - t2) / (K - 2) if K > 2 else tv / K  # the state-step kernel
            mv = cells * K / tv / 1e6
            variants[storage] = {"mlups": round(mv, 1), "steps": K, "bytes_per_cell": 76,
                                 "rounding": "stochastic (cvt.rs)",
                                 "over_fp32": round(mv / (mlups / world), 3),
                                 "state_step_ms": round(tk * 1e3, 4),
                                 "state_step_mlups": round(cells / tk / 1e6, 1),
                                 "state_step_over_fp32": round(t_kernel / tk, 3),
                                 "hbm_frac": round(cells * 76 / tk / 1e9 / _peaks()[0], 4),
                                 "hbm_frac_whole_rollout": round(mv * 1e6 * 76 / 1e9
                                                                 / _peaks()[0], 4)}
            del vn, vs
        torch.cuda.empty_cache()

    if not args.no_variants and rank == 0:
        # shorter measurements first; the 512^3 precision study (tens of seconds
        # at the power cap) last, so that its heat does not slow the others
        variants["batched"] = batched_cost(dev)
        torch.cuda.empty_cache()
        variants["adjoint"] = adjoint_cost(dev)
        torch.cuda.empty_cache()
        variants["pipe"] = pipe_cost(dev)
        torch.cuda.empty_cache()
        variants["d2q9"] = d2q9_cost(dev)
        torch.cuda.empty_cache()
        variants["c1"] = c1_cost(dev)
        torch.cuda.empty_cache()
        variants["frames"] = frames_cost(dev)
        torch.cuda.empty_cache()
        variants["sharded"] = sharded_cost(dev)
        torch.cuda.empty_cache()
        variants["precision_512"] = precision_cost(dev, args.c5_steps)

    upd = update_call_cost(dev) if (rank == 0 and not args.no_variants) else None
    if rank == 0:
        peak, peak_kind = _peaks()
        achieved = bytes_per_cell * cells / t_kernel / 1e9  # per GPU
        line = {
            "metric": METRIC, "value": round(mlups, 1), "unit": "MLUPS",
            "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": round(t_dev / K * 1e3, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.storage == "f64" else "f32",
            "data": "synthetic (seeded spheres, rng seed 0)",
            "config": {"workload": WORKLOAD, "grid": list(GRID), "lattice": "D3Q19",
                       "storage": f"{args.storage} offsets", "tau": TAU, "solid_fraction": float(wall.mean()),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "state 2 x 1.27 GB > 126 MB L2; no flush needed"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1),
                         "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "peak_source": peak_kind,
                         "traffic": (NCU_TRAFFIC_256_F32 if GRID == (256, 256, 256)
                                     and args.storage == "f32" else None),
                         "traffic_unit": "DRAM bytes per launch (ncu)",
                         "algorithmic_bytes_per_launch": bytes_per_cell * cells,
                         "bytes_per_cell": bytes_per_cell,
                         "kernel": KERNEL_LABEL[args.storage],
                         "kernel_ms": round(t_kernel * 1e3, 4),
                         "kernel_ms_how": "CUDA events: (t(K-step rollout) - t(2-step "
                                          "rollout)) / (K - 2)",
                         "whole_rollout_frac": round(bytes_per_cell * cells * K / t_dev / 1e9
                                                     / peak, 4)},
            "e2e": {"value": round(_job_mlups(world, cells, K, t_e2e), 1), "unit": "MLUPS",
                    "h2d_bytes_per_step": h2d // K, "d2h_bytes_per_step": d2h // K,
                    "note": "LBMNode.run with pinned-host state in/out, per K-step rollout"},
            # the first step (one-pass tiled kernel), K - 2 state steps, the last step
            "gpu_launches": K,
            "clocks": clocks,
            "update_call": upd,
            "host": host_info(),
            "variants": variants,
        }
        if world == 1 and not args.no_cpu_baseline:
            procs = _host_cores()
            v, _ = cpu_baseline(procs, nx=16, steps=4)
            line["cpu_baseline"] = {"value": round(v, 3), "unit": "MLUPS", "cores": procs,
                                    "kind": "port",
                                    "sample": f"{procs} processes x 16x256x256 slab of the "
                                              "workload x 4 steps (float32 restatement of "
                                              "the reference step; JAX absent)"}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def precision_cost(dev, steps):
    """512^3 D3Q19 obstacle flow (the 256^3 workload's generator: spheres of
    radii 4-12, 10 % solid; velocity inlet 0.05, zero-gradient outlet, tau 0.6),
    `steps` steps with populations stored as FP64 (the reference run, FP64
    arithmetic), FP32, FP16 and BF16 offsets (FP32 arithmetic).  Reports MLUPS
    of each and the relative L2 error of density, density - 1 and velocity
    against the FP64 run, computed on the device."""
    import torch
    from maddening_b200 import LBMNode
    from maddening_b200.geometry import random_spheres
    grid = (512, 512, 512)
    cells = grid[0] * grid[1] * grid[2]
    wall = random_spheres(grid, seed=0)
    bi = {"inlet_velocity": np.array(U_IN)}
    out, ref = {}, None

    def rel(a, b):
        return float(torch.linalg.vector_norm((a.double() - b).flatten())
                     / torch.linalg.vector_norm(b.flatten()))

    for storage in ("f64", "f32", "f16", "bf16"):
        node = LBMNode("p", 1.0, grid_shape=grid, viscosity=(TAU - 0.5) / 3.0, wall_mask=wall,
                       outlet_condition="zero_gradient", storage=storage, device=dev)
        st = node.initial_state()
        node.run(st, bi, 2)  # warm-up
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        res = node.run(st, bi, steps)
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        entry = {"mlups": round(cells * steps / t / 1e6, 1)}
        rho, vel = res["density"], res["velocity"]
        del res, st, node
        torch.cuda.empty_cache()
        if storage == "f64":
            ref = (rho, vel)
        else:
            entry["relL2_rho"] = float(f"{rel(rho, ref[0]):.3e}")
            entry["relL2_rho_minus_1"] = float(f"{rel(rho - 1.0, ref[0] - 1.0):.3e}")
            entry["relL2_u"] = float(f"{rel(vel, ref[1]):.3e}")
            del rho, vel
        out[storage] = entry
    for storage in ("f16", "bf16"):
        out[storage]["over_fp32"] = round(out[storage]["mlups"] / out["f32"]["mlups"], 3)
    del ref
    torch.cuda.empty_cache()
    return {"workload": f"512^3 D3Q19 obstacle flow, {steps} steps, errors vs the FP64 "
                        "storage run", **out}


def batched_cost(dev, steps=500):
    """64 uneven D3Q19 lattices (extents log-uniform in [32, 160], tau in
    [0.55, 1.5], z walls, g_x in [1e-7, 1e-5]), 500 steps: one autotuned batched
    launch per step (FP32 and FP16 storage) against one plain rollout per
    instance (FP32 storage, and FP16 for reference); best of three runs of
    each arm."""
    import torch
    from maddening_b200.batched import LBMEnsemble, uneven_ensemble
    out = {"workload": "64 uneven D3Q19 lattices, 500 steps"}
    for storage in ("f32", "f16"):
        nodes, bis = uneven_ensemble(64, seed=0, storage=storage, device=dev)
        states = [n.initial_state() for n in nodes]
        ens = LBMEnsemble(nodes)
        cfg = ens.autotune(states, bis, n_steps=10, use_cache=False)
        ws = torch.empty(ens.workspace_bytes(), dtype=torch.uint8, device=dev)
        ens.run(states, bis, 3, workspace=ws)
        for n, st, bi in zip(nodes, states, bis):
            n.run(st, bi, 3)
        torch.cuda.synchronize()
        # each arm three times, best of each (the same for both arms)
        t_b = t_p = float("inf")
        for _ in range(3):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record()
            ens.run(states, bis, steps, workspace=ws)
            e[1].record()
            e[2].record()
            for n, st, bi in zip(nodes, states, bis):
                n.run(st, bi, steps)
            e[3].record()
            torch.cuda.synchronize()
            t_b = min(t_b, e[0].elapsed_time(e[1]) / 1e3)
            t_p = min(t_p, e[2].elapsed_time(e[3]) / 1e3)
        cells = ens.cells
        out["cells"] = cells
        out[f"batched_{storage}_mlups"] = round(cells * steps / t_b / 1e6, 1)
        out[f"plain_{storage}_per_instance_mlups"] = round(cells * steps / t_p / 1e6, 1)
        out[f"config_{storage}"] = cfg
        del ens, states, ws, nodes
        torch.cuda.empty_cache()
    ref = out["plain_f32_per_instance_mlups"]
    out["batched_f32_over_plain_f32"] = round(out["batched_f32_mlups"] / ref, 3)
    out["batched_f16_over_plain_f32"] = round(out["batched_f16_mlups"] / ref, 3)
    out["hbm_frac_batched_f32"] = round(out["batched_f32_mlups"] * 1e6 * 152 / 1e9 / _peaks()[0], 4)
    out["hbm_frac_batched_f16"] = round(out["batched_f16_mlups"] * 1e6 * 76 / 1e9 / _peaks()[0], 4)
    return out


def pipe_cost(dev, steps=200, grid=(384, 192, 192)):
    """The pipe node (LBMPipeNode) on a 384 x 192 x 192 pipe (14.2 M cells,
    radius 0.9, propeller disc at x = nx / 4), FP32, best of three K-step runs of
    ``run`` (populations in and out in the reference layout):
    single phase (propeller 4e-4, gravity -1e-5, 70% fill) and Shan-Chen
    multiphase (G = -4.5, liquid 1.3 / gas 0.3, half filled).  Bytes per cell
    and step of the passes as built: single phase 152 (D3Q19) + 56 (D3Q7
    tracer) = 208 in one fused pass; multiphase 76 + 4 (density pass) + 76 + 4
    + 76 (collide: pull, psi of the neighbours, aligned store) = 236."""
    import torch
    from maddening_b200.pipe import LBMPipeNode
    nx, ny, nz = grid
    out = {"workload": "%dx%dx%d pipe, FP32, %d steps" % (nx, ny, nz, steps)}
    kw = dict(nx=nx, ny=ny, nz=nz, tau=0.8, pipe_radius=0.9, propeller_x=nx // 4,
              propeller_radius=0.8, propeller_strength=4e-4, initial_velocity=0.005,
              gravity=-1e-5, tau_tracer=0.6)
    modes = {"single_phase": (dict(fill_fraction=0.7), 208),
             "multiphase": (dict(fill_fraction=0.5, G=-4.5, rho_liquid=1.3, rho_gas=0.3), 236)}
    for name, (extra, bpc) in modes.items():
        node = LBMPipeNode("bench_pipe", 1.0, device=dev, **kw, **extra)
        st = node.initial_state()
        node.run(st, {}, 3)
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(3):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            node.run(st, {}, steps)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        cells = nx * ny * nz
        m = cells * steps / best / 1e6
        out[name] = {"mlups": round(m, 1), "bytes_per_cell": bpc,
                     "hbm_frac": round(m * 1e6 * bpc / 1e9 / _peaks()[0], 4)}
        del node, st
        torch.cuda.empty_cache()
    return out


def d2q9_cost(dev, grid=(4096, 4096), steps=500):
    """D2Q9 channel: 4096 x 4096 (16.8 M cells), walls on the two y rows,
    periodic x, uniform force 1e-6 along x, tau 0.6; FP32 (72 B per cell and
    step) and FP16 offsets (36 B); best of three K-step rollouts."""
    import torch
    from maddening_b200 import LBMNode
    wall = np.zeros(grid, dtype=bool)
    wall[:, 0] = wall[:, -1] = True
    bi = {"body_force": np.array([1e-6, 0.0], dtype=np.float32)}
    cells = grid[0] * grid[1]
    out = {"workload": "%dx%d D2Q9 channel, %d steps" % (grid[0], grid[1], steps)}
    for storage, bpc in (("f32", 72), ("f16", 36)):
        node = LBMNode("d2", 1.0, grid_shape=grid, viscosity=(TAU - 0.5) / 3.0, lattice="D2Q9",
                       wall_mask=wall, storage=storage, device=dev)
        st = node.initial_state()
        node.run(st, bi, 3)
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(3):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            node.run(st, bi, steps)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        m = cells * steps / best / 1e6
        out[storage] = {"mlups": round(m, 1), "bytes_per_cell": bpc,
                        "hbm_frac": round(m * 1e6 * bpc / 1e9 / _peaks()[0], 4)}
        del node, st
        torch.cuda.empty_cache()
    out["f16_over_f32"] = round(out["f16"]["mlups"] / out["f32"]["mlups"], 3)
    return out


def c1_cost(dev, grid=(64, 64, 64), steps=500):
    """The 64^3 channel (z walls, periodic x and y, tau 0.8, body force 1e-6 x,
    FP32), 500 steps: a rollout as queued launches, and the same rollout
    captured once in a CUDA graph and replayed.  Its 40 MB of state stay in the
    126 MB L2, so the HBM fraction is indicative only; launch gaps dominate."""
    import torch
    from maddening_b200 import LBMNode
    wall = np.zeros(grid, dtype=bool)
    wall[:, :, 0] = wall[:, :, -1] = True
    node = LBMNode("c1", 1.0, grid_shape=grid, viscosity=0.1, wall_mask=wall, device=dev)
    bi = {"body_force": np.array([1e-6, 0.0, 0.0], dtype=np.float32)}
    st = node.initial_state()
    cells = grid[0] * grid[1] * grid[2]

    def timed(fn):
        best = float("inf")
        for _ in range(5):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        return cells * steps / best / 1e6

    node.run(st, bi, 3)
    torch.cuda.synchronize()
    plain = timed(lambda: node.run(st, bi, steps))
    out = {"workload": "64^3 channel, z walls, force, FP32, %d steps" % steps,
           "queued_mlups": round(plain, 1)}
    try:
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            node.run(st, bi, steps)
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            node.run(st, bi, steps)
        g.replay()
        torch.cuda.synchronize()
        out["graph_mlups"] = round(timed(g.replay), 1)
        del g
    except Exception as exc:  # capture needs no host sync inside run
        out["graph_mlups"] = None
        out["graph_error"] = str(exc)[:200]
    out["bytes_per_cell"] = 152
    best = max(v for v in (out["queued_mlups"], out.get("graph_mlups") or 0))
    out["hbm_frac_indicative"] = round(best * 1e6 * 152 / 1e9 / _peaks()[0], 4)
    return out


def update_call_cost(dev, grid=(256, 256, 256), calls=40):
    """One ``LBMNode.update`` call per step, as a graph manager drives the node
    (the reference-layout state in and out of every call), on the benchmark
    workload; mean over ``calls`` calls issued from Python, and over the same
    calls captured once in a CUDA graph and replayed (``graph_ms_per_call``).  The default one-pass tiled kernel
    moves 173 B per cell (f in 76, wall 1, f out 76, density + velocity +
    pressure 20); the two-pass form (collide into the workspace, then the pull
    step) moves 324 and is timed beside it."""
    import torch
    from maddening_b200 import LBMNode
    from maddening_b200.geometry import random_spheres
    wall = random_spheres(grid, seed=0)
    bi = {"inlet_velocity": np.array(U_IN)}
    cells = grid[0] * grid[1] * grid[2]
    res = {"workload": "LBMNode.update, one call per step, %s" % "x".join(map(str, grid))}
    for one_pass in (True, False):
        node = LBMNode("call", 1.0, grid_shape=grid, viscosity=(TAU - 0.5) / 3.0,
                       wall_mask=wall, outlet_condition="zero_gradient", device=dev,
                       one_pass=one_pass)
        st = node.initial_state()
        for _ in range(3):
            st = node.update(st, bi, 1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev) as clk:  # the one pass is SM-bound: its time follows the clock
            e0.record()
            for _ in range(calls):
                st = node.update(st, bi, 1.0)
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / calls
        sm = clk.summary()
        # the same calls replayed from a CUDA graph: the device time per call
        # without the Python side of update (which can fall behind a fast call)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            node.update(st, bi, 1.0)
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        s_in = st
        with torch.cuda.graph(g):
            for _ in range(calls):
                s_in = node.update(s_in, bi, 1.0)
        g.replay()
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record()
        g.replay()
        g1.record()
        torch.cuda.synchronize()
        ms_graph = g0.elapsed_time(g1) / calls
        del g, s_in
        bpc = 173 if one_pass else 324
        frac = round(cells * bpc / (ms * 1e-3) / 1e9 / _peaks()[0], 4)
        if one_pass:
            res.update({"value": round(cells / ms / 1e3, 1), "unit": "MLUPS",
                        "ms_per_call": round(ms, 4), "bytes_per_cell": bpc, "hbm_frac": frac,
                        "kernel": "k_tiled<19,float,kOutAoS,faces,no force> (one pass)",
                        "sm_mhz": sm.get("sm_mhz"), "clock_reasons": sm.get("reasons"),
                        "graph_ms_per_call": round(ms_graph, 4),
                        "graph_mlups": round(cells / ms_graph / 1e3, 1)})
        else:
            res["two_pass"] = {"value": round(cells / ms / 1e3, 1), "ms_per_call": round(ms, 4),
                               "bytes_per_cell": bpc, "hbm_frac": frac, "sm_mhz": sm.get("sm_mhz"),
                               "graph_ms_per_call": round(ms_graph, 4)}
        del node, st
        torch.cuda.empty_cache()
    return res


def sharded_cost(dev, grid=(256, 256, 256), steps=20):
    """The slab-sharded runner (``ShardedLBM``) with one rank on this GPU: the
    256^3 lattice with the benchmark's spheres and a body force along x (no
    faces: the sharded axis 0 carries none), FP32; per step one state step of
    the padded slab and the pad refresh of the 5 crossing populations of each
    face, issued from Python.  Timed beside ``LBMNode.run`` of the same lattice
    (CUDA events, best of three)."""
    import torch
    from maddening_b200 import LBMNode
    from maddening_b200.geometry import random_spheres
    from maddening_b200.sharded import ShardedLBM
    cells = grid[0] * grid[1] * grid[2]
    node = LBMNode("sharded", 1.0, grid_shape=grid, viscosity=(TAU - 0.5) / 3.0,
                   wall_mask=random_spheres(grid, seed=0), device=dev)
    bi = {"body_force": np.array([1e-6, 0.0, 0.0], dtype=np.float32)}
    st = node.initial_state()
    sh = ShardedLBM(node)
    sh.scatter(st)
    sh.run(bi, 3)

    def best(fn):
        t = float("inf")
        for _ in range(3):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            t = min(t, e0.elapsed_time(e1))
        return t

    t_sh = best(lambda: sh.run(bi, steps))
    node.run(st, bi, 3)
    t_run = best(lambda: node.run(st, bi, steps))
    del sh
    return {"workload": "%s spheres + body force, FP32, %d steps, one rank"
                        % ("x".join(map(str, grid)), steps),
            "sharded_mlups": round(cells * steps / t_sh / 1e3, 1),
            "run_mlups": round(cells * steps / t_run / 1e3, 1),
            "sharded_over_run": round(t_run / t_sh, 3),
            "note": "node.run includes its first collide from the reference layout and the "
                    "last step back to it; the sharded steps stay in the state layout"}


def frames_cost(dev, grid=(256, 256, 256), frames=20):
    """Streaming frames of a running node (BinaryStateEncoder over density and
    velocity of the benchmark lattice, 16 B per cell): the one-launch device
    gather alone (encode_device) and whole frames to host bytes (encode)."""
    import torch
    from maddening_b200 import LBMNode
    from maddening_b200.streaming import BinaryStateEncoder
    node = LBMNode("frames", 1.0, grid_shape=grid, viscosity=(TAU - 0.5) / 3.0, device=dev)
    st = node.run(node.initial_state(), {"body_force": np.array([1e-6, 0.0, 0.0])}, 3)
    state = {"vessel": st}
    enc = BinaryStateEncoder(state, fields={"vessel": ["density", "velocity"]})
    enc.encode(0.0, state)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(frames):
        enc.encode_device(state)
    e1.record()
    torch.cuda.synchronize()
    t_pack = e0.elapsed_time(e1) / frames / 1e3
    t0 = time.perf_counter()
    for i in range(frames):
        frame = enc.encode(float(i), state)
    t_frame = (time.perf_counter() - t0) / frames
    t0 = time.perf_counter()
    for i in range(frames):
        enc.encode_view(float(i), state)
    t_view = (time.perf_counter() - t0) / frames
    payload = enc.total_floats * 4
    return {"workload": "frames of density + velocity, %s lattice" % "x".join(map(str, grid)),
            "frame_bytes": len(frame), "pack_ms": round(t_pack * 1e3, 4),
            "pack_hbm_frac": round(2 * payload / t_pack / 1e9 / _peaks()[0], 4),
            "frame_ms": round(t_frame * 1e3, 3),
            "frame_gbs": round(len(frame) / t_frame / 1e9, 2),
            "view_ms": round(t_view * 1e3, 3),
            "view_gbs": round(len(frame) / t_view / 1e9, 2),
            "note": "frame: pack + one device-to-host copy into the pinned frame buffer + one "
                    "copy into bytes; view: the same without the bytes copy"}


def adjoint_cost(dev):
    """Cost of the differentiated rollout against the plain forward: 128^3 D3Q19,
    z walls, tau 0.7, force field 1e-6 N(0,1), 1000 steps, checkpoint every 32,
    loss = final kinetic energy (FP32 storage)."""
    import torch
    from maddening_b200 import LBMNode
    from maddening_b200.geometry import z_walls
    grid, steps, K = (128, 128, 128), 1000, 32
    rng = np.random.default_rng(0)
    node = LBMNode("adj", 1.0, grid_shape=grid, viscosity=0.2 / 3.0, wall_mask=z_walls(grid),
                   device=dev)
    st = node.initial_state()
    F = torch.tensor(1e-6 * rng.standard_normal(grid + (3,)), dtype=torch.float32, device=dev,
                     requires_grad=True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    node.run(st, {"body_force": F.detach()}, 10)
    warm = node.rollout(st, {"body_force": F}, steps, checkpoint_every=K)  # allocations
    (0.5 * (warm["density"] * (warm["velocity"] ** 2).sum(-1)).sum()).backward()
    F.grad = None
    del warm
    torch.cuda.synchronize()
    ev[0].record()
    node.run(st, {"body_force": F.detach()}, steps)
    ev[1].record()
    ev[2].record()
    out = node.rollout(st, {"body_force": F}, steps, checkpoint_every=K)
    loss = 0.5 * (out["density"] * (out["velocity"] ** 2).sum(-1)).sum()
    ev[3].record()
    ev[4].record()
    loss.backward()
    ev[5].record()
    torch.cuda.synchronize()
    t_plain = ev[0].elapsed_time(ev[1])
    t_fwd = ev[2].elapsed_time(ev[3])
    t_bwd = ev[4].elapsed_time(ev[5])
    return {"workload": "128^3 D3Q19, z walls, tau 0.7, force field, 1000 steps, "
                        "checkpoint every 32, FP32",
            "plain_forward_ms": round(t_plain, 2), "checkpointed_forward_ms": round(t_fwd, 2),
            "backward_ms": round(t_bwd, 2),
            "backward_over_forward": round(t_bwd / t_plain, 3),
            "forward_plus_backward_over_forward": round((t_fwd + t_bwd) / t_plain, 3),
            "workspace_gb": round(node.plan.adjoint_workspace_bytes(steps, K) / 1e9, 2)}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    procs = _host_cores()
    # each step: every process advances a 16x256x256 slab of the workload by
    # one step; W and K are bounded (3 and 8) so the run takes well under a minute
    warm = min(max(args.warmup, 3), 3)
    steps = max(1, min(args.steps, 8))
    cpu_baseline(procs, nx=16, steps=warm)
    v, wall_s = cpu_baseline(procs, nx=16, steps=steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "MLUPS",
        "n_gpus": world, "steps": steps, "warmup": warm, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded spheres, rng seed 0)",
        "config": {"workload": WORKLOAD, "grid": list(GRID)},
        "cpu_baseline": {"value": round(v, 3), "unit": "MLUPS", "cores": procs, "kind": "port",
                         "sample": f"{procs} processes x 16x256x256 slab x {steps} steps "
                                   "(float32 restatement of the reference step; JAX absent)"},
        "e2e": {"value": round(v, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "host": host_info(),
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--storage", choices=["f32", "f16", "bf16", "f64"], default="f32",
                    help="population storage of the measured run (default f32)")
    ap.add_argument("--grid", type=int, default=256,
                    help="cube side (256 = the benchmark workload; smaller for profiling)")
    ap.add_argument("--c5-steps", type=int, default=2000,
                    help="steps of the 512^3 precision comparison (variants)")
    ap.add_argument("--only", choices=["pipe", "update_call", "frames", "d2q9", "c1", "batched",
                                       "sharded"],
                    help="run one variant alone and print its JSON (for profiling)")
    ap.add_argument("--variant-grid", default=None,
                    help="lattice of --only, e.g. 192x128x128 (default: the variant's own)")
    args = ap.parse_args()
    global GRID
    GRID = (args.grid,) * 3
    if args.warmup < 3:
        args.warmup = 3
    if args.only:
        import torch
        dev = torch.device("cuda", 0)
        kw = {}
        if args.variant_grid and args.only != "batched":
            kw["grid"] = tuple(int(v) for v in args.variant_grid.split("x"))
        fn = {"pipe": pipe_cost, "update_call": update_call_cost, "frames": frames_cost,
              "d2q9": d2q9_cost, "c1": c1_cost, "batched": batched_cost,
              "sharded": sharded_cost}[args.only]
        if args.only == "pipe":
            kw["steps"] = args.steps
        print(json.dumps({args.only: fn(dev, **kw)}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
