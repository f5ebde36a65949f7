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
