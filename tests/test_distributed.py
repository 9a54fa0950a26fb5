"""CPU tests of replica sharding: the partition is balanced and complete,
and run_sharded gathers every replica's result in spec order across two
gloo ranks (the runner is a CPU stand-in; no GPU work here)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from chllmodel_b200.batched import phase_grid
from chllmodel_b200.distributed import run_sharded, shard


def _specs():
    return phase_grid([0.1, 0.5, 1.0, 2.0], [0.0, 1.0, 2.0, 3.0], [32, 48, 64], K=1.0, seed=1,
                      size_seed=12345)


def test_shard_is_a_balanced_partition():
    specs = _specs()
    for world in (1, 2, 3, 8):
        parts = shard(specs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(specs)))
        loads = [sum(specs[i]["ni"] ** 3 for i in p) for p in parts]
        biggest = max(s["ni"] ** 3 for s in specs)
        assert max(loads) - min(loads) <= biggest
    assert shard(specs, 2) == shard(specs, 2)


def _fake_runner(share):
    return [{"kT": s["kT"], "g": s["g"], "n": s["ni"] * s["nj"] * s["nk"]} for s in share]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = run_sharded(_specs(), _fake_runner, rank, world)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(120)
def test_run_sharded_gathers_in_order_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world = 2
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=100) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert got[1] is None
    specs = _specs()
    assert got[0] == _fake_runner(specs)
