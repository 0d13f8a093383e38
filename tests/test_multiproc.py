"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): each rank takes its own
shard of the case stream (replicas, weak scaling), shards are disjoint and cover the stream,
and the step time reported is the maximum over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, batch, steps, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    mine = []
    for s in range(steps):
        start = ((s * world + rank) * batch) % bench.TOTAL_CASES
        mine.extend(range(start, start + batch))
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((gathered, float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_and_max_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    world, batch, steps = 2, 7, 3
    procs = [ctx.Process(target=_worker, args=(r, world, port, batch, steps, out)) for r in range(world)]
    for p in procs:
        p.start()
    gathered, tmax = out.get(timeout=120)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    a, b = set(gathered[0]), set(gathered[1])
    assert not (a & b)
    assert a | b == set(range(world * batch * steps))
    assert tmax == 2.0


def test_step_cases_shards_are_deterministic():
    import bench
    x = [c[1].tobytes() for c in bench.step_cases(1, 0, 2, 3, config=1)]
    y = [c[1].tobytes() for c in bench.step_cases(1, 0, 2, 3, config=1)]
    z = [c[1].tobytes() for c in bench.step_cases(1, 1, 2, 3, config=1)]
    assert x == y and x != z
