"""The N > 1 path of bench.py on CPU: world-size-2 gloo ranks run independent replicas (no
data-path collective) and agree on the max-over-ranks time used for the whole-job value."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    w, r, lr = bench.dist_setup()
    dist.init_process_group("gloo", rank=r, world_size=w)
    try:
        # each rank owns its own replica (seed = 2 + rank), the only collective is the timing max
        ms = 10.0 + 5.0 * rank
        t = torch.tensor([ms], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        cfg = bench.config_dict(type("A", (), {"n": 16, "tsteps": 2, "gpus": w})())
        q.put((r, w, float(t.item()), cfg["parallelism"]))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(world))
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2 and o[2] == 15.0 and o[3] == "replicas2" for o in out)


def _slab_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from set_b200 import slab as SL
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nz, ps = 11, 6
        glob = torch.arange(8 * nz * ps, dtype=torch.float64).reshape(8, nz, ps)
        k0, n = SL.split_z(nz, world)[rank]
        X = torch.full((8, n + 2 * SL.GHOST, ps), float("nan"), dtype=torch.float64)
        X[:, SL.GHOST:SL.GHOST + n] = glob[:, k0:k0 + n]
        SL.exchange_halos(X, n, rank, world)
        lo = X[:, 0:SL.GHOST]
        hi = X[:, n + SL.GHOST:]
        ok_lo = torch.isnan(lo).all().item() if rank == 0 else torch.equal(lo, glob[:, k0 - SL.GHOST:k0])
        ok_hi = (torch.isnan(hi).all().item() if rank == world - 1
                 else torch.equal(hi, glob[:, k0 + n:k0 + n + SL.GHOST]))
        own = torch.equal(X[:, SL.GHOST:SL.GHOST + n], glob[:, k0:k0 + n])
        dt = torch.tensor([0.5 + 0.1 * ((rank * 7) % world)], dtype=torch.float64)
        SL.min_dt(dt)
        q.put((rank, bool(ok_lo), bool(ok_hi), bool(own), float(dt.item())))
    finally:
        dist.destroy_process_group()


def test_slab_halo_exchange_three_ranks_gloo():
    """The z-slab exchange on CPU tensors: every interior ghost plane receives the neighbour's
    owned edge plane, the grid's end ghosts are left alone, owned planes are untouched, and the
    next step's dt becomes the minimum over ranks."""
    world, port = 3, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_slab_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(world))
    assert [o[0] for o in out] == [0, 1, 2]
    assert all(o[1] and o[2] and o[3] for o in out), out
    assert all(o[4] == 0.5 for o in out)
