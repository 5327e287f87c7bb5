"""The N > 1 path (replicas only) with two gloo ranks on the CPU: problem
sharding covers every problem exactly once with balanced loads, and the timing
aggregate is the max over ranks with cell-steps summed."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import cases
import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [c["nx"] * c["ny"] for c in cases.ensemble(seed=3, n=40)]
        mine = replicas.shard(sizes, rank, world)
        local_ms = 10.0 + 5.0 * rank
        local_cells = float(sum(sizes[i] for i in mine))
        ms, cells = replicas.aggregate(local_ms, local_cells, dist, device="cpu")
        q.put((rank, mine, ms, cells, sum(sizes)))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    idx = sorted(out[0][1] + out[1][1])
    assert idx == list(range(40))
    assert not set(out[0][1]) & set(out[1][1])
    for _, _, ms, cells, total in out:
        assert ms == 15.0 and cells == total
    sizes = [c["nx"] * c["ny"] for c in cases.ensemble(seed=3, n=40)]
    loads = [sum(sizes[i] for i in o[1]) for o in out]
    assert max(loads) / min(loads) < 1.2


def test_shard_single_rank_takes_all():
    assert replicas.shard([5, 3, 9], 0, 1) == [0, 1, 2]
