"""Halo refresh of the slab-sharded runner on CPU (gloo): after ``fill_halos``
every rank's padded block equals the global lattice's periodic neighbourhood
of its slab -- the halo planes of axis 0 from the neighbouring ranks (two
ranks: the same peer on both sides; three: distinct peers), the halos of the
other axes by periodic copies, corners included."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from maddening_b200.sharded import fill_halos


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _expected(g, lo, n0):
    idx0 = np.arange(lo - 1, lo + n0 + 1) % g.shape[0]
    blk = np.take(g, idx0, axis=0)
    for ax in range(1, g.ndim - 1):
        blk = np.take(blk, np.arange(-1, g.shape[ax] + 1) % g.shape[ax], axis=ax)
    return blk


def _block(g, lo, n0):
    pad = [(1, 1)] * (g.ndim - 1) + [(0, 0)]
    return torch.from_numpy(np.pad(g[lo: lo + n0], pad).copy())


def _rank(rank, world, port, shape, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        g = np.random.default_rng(0).standard_normal(shape).astype(np.float32)
        n0 = shape[0] // world
        fp = _block(g, rank * n0, n0)
        fill_halos(fp, rank, world)
        out.put((rank, bool(np.array_equal(fp.numpy(), _expected(g, rank * n0, n0)))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,shape", [(2, (6, 5, 4, 19)), (3, (9, 4, 3, 19)), (2, (4, 7, 9))])
def test_halos_match_the_global_lattice(world, shape):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, shape, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(r, True) for r in range(world)]


def test_single_rank_wraps_locally():
    g = np.random.default_rng(1).standard_normal((5, 4, 6, 19)).astype(np.float32)
    fp = _block(g, 0, 5)
    fill_halos(fp, 0, 1)
    assert np.array_equal(fp.numpy(), _expected(g, 0, 5))
