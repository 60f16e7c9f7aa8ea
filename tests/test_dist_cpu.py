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
