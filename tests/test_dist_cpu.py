"""The multi-rank bench path on CPU (gloo, world size 2): ranks are independent
replicas with no data-path collective; the barrier, the max-over-ranks timing
and the whole-job aggregate are the only cross-rank steps, and under torchrun
only rank 0 runs and prints the reference arm."""

import io
import os
import socket
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        bench._barrier(world)
        t = bench._max_over_ranks(world, 0.25 + 0.5 * rank)  # rank 1 is the slow one
        out.put((rank, t, bench._job_mlups(world, 1000, 10, t)))
        bench._barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [0.75, 0.75]
    # 2 replicas x 1000 cells x 10 steps in 0.75 s
    assert res[0][2] == pytest.approx(2 * 1000 * 10 / 0.75 / 1e6)


def test_single_rank_needs_no_collective():
    assert bench._max_over_ranks(1, 0.5) == 0.5
    assert bench._job_mlups(1, 16_777_216, 1000, 0.4) == pytest.approx(41943.04)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(type("A", (), {"warmup": 3, "steps": 2})())
    assert buf.getvalue() == ""


def test_reference_arm_line_on_rank_zero(monkeypatch):
    """Rank 0 prints one JSON line for the CPU port: bounded warm-up (>= 3) and
    timed steps, the measured value repeated as cpu_baseline and e2e."""
    import json
    calls = []

    def fake_cpu_baseline(procs, nx, steps):
        calls.append(steps)
        return 3.5, 1.0

    monkeypatch.setenv("WORLD_SIZE", "1")
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setattr(bench, "cpu_baseline", fake_cpu_baseline)
    monkeypatch.setattr(bench, "_host_cores", lambda: 4)
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(type("A", (), {"warmup": 10, "steps": 1000})())
    line = json.loads(buf.getvalue())
    assert calls == [3, 8]
    assert line["impl"] == "reference" and line["warmup"] == 3 and line["steps"] == 8
    assert line["value"] == line["cpu_baseline"]["value"] == line["e2e"]["value"] == 3.5
    assert line["cpu_baseline"]["cores"] == 4 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
