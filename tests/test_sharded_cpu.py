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


def _rank_slices(rank, world, port, q, n, sl, out):
    import torch.distributed as dist
    from datetime import timedelta
    from maddening_b200.lattice import by_name
    from maddening_b200.sharded import crossing_populations, exchange_slices
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        lat = by_name("D3Q19" if q == 19 else "D2Q9")
        plus, minus = crossing_populations(lat)
        # every rank's state: interior slices from a global array, pads junk
        g = np.random.default_rng(0).standard_normal((q, world * n, sl)).astype(np.float32)
        st = np.full((q, n + 2, sl), np.nan, dtype=np.float32)
        st[:, 1:-1] = g[:, rank * n:(rank + 1) * n]
        t = torch.from_numpy(st.copy())
        exchange_slices(t, plus, minus, rank, world, staged=True)
        res = t.numpy()
        ok = np.array_equal(res[:, 1:-1], st[:, 1:-1])  # interior untouched
        prev_last = g[:, (rank * n - 1) % (world * n)]
        next_first = g[:, ((rank + 1) * n) % (world * n)]
        ok &= np.array_equal(res[plus, 0], prev_last[plus])
        ok &= np.array_equal(res[minus, -1], next_first[minus])
        others = [i for i in range(q) if i not in plus]
        ok &= bool(np.isnan(res[others, 0]).all())  # only the crossing ones are sent
        out.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,q,n,sl", [(2, 19, 3, 20), (3, 19, 2, 12), (2, 9, 4, 7)])
def test_exchange_sends_only_crossing_populations(world, q, n, sl):
    """The state-layout runner's exchange: pad slice 0 receives the +1
    populations (5 of D3Q19, 3 of D2Q9) of the previous rank's last slice, pad
    slice n + 1 the -1 populations of the next rank's first slice, nothing
    else moves (gloo, 2 and 3 ranks)."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_slices, args=(r, world, port, q, n, sl, out))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(r, True) for r in range(world)]


def test_crossing_populations_of_both_lattices():
    from maddening_b200.lattice import by_name
    from maddening_b200.sharded import crossing_populations
    for name, n in (("D3Q19", 5), ("D2Q9", 3)):
        lat = by_name(name)
        plus, minus = crossing_populations(lat)
        assert len(plus) == len(minus) == n
        e = np.asarray(lat.e)
        assert all(e[q, 0] == 1 for q in plus) and all(e[q, 0] == -1 for q in minus)
