"""CPU tests of the z-slab plumbing: the plane partition, and TorchHalo's halo
exchange and count all-reduce across gloo ranks (host tensors stand in for a
slab's planes; the GPU test of the same sweep on one device is
test_slab_gpu.py)."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from chllmodel_b200.slab import FIRST_OWN, LAST_OWN, LOWER_HALO, UPPER_HALO, TorchHalo, \
    neighbours, split_planes

PLANE = 6  # floats per fake plane


def test_slab_neighbours():
    """Below/above of each slab: every slab's upper neighbour has it as its
    lower one (the halo written and the halo read are the same pair)."""
    assert neighbours(0, 1, True) == (0, 0)
    assert neighbours(0, 1, False) == (None, None)
    assert neighbours(0, 2, True) == (1, 1)
    assert [neighbours(r, 3, False) for r in range(3)] == [(None, 1), (0, 2), (1, None)]
    for n in (1, 2, 3, 5):
        for periodic in (False, True):
            for r in range(n):
                down, up = neighbours(r, n, periodic)
                if up is not None:
                    assert neighbours(up, n, periodic)[0] == r
                if down is not None:
                    assert neighbours(down, n, periodic)[1] == r


def test_split_planes():
    for nk, parts in [(16, 2), (16, 3), (480, 8), (10, 5), (12, 1)]:
        out = split_planes(nk, parts)
        assert [z0 for z0, _ in out] == [sum(n for _, n in out[:r]) for r in range(parts)]
        assert sum(n for _, n in out) == nk
        assert all(n % 2 == 0 and n >= 2 for _, n in out)
        assert max(n for _, n in out) - min(n for _, n in out) <= 2
    with pytest.raises(ValueError):
        split_planes(15, 2)
    with pytest.raises(ValueError):
        split_planes(8, 5)


def _pattern(rank, colour, which):
    return torch.full((PLANE,), 1000.0 * rank + 10.0 * colour + which)


def _worker(rank, world, periodic, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        planes = {(c, w): (_pattern(rank, c, w) if w in (FIRST_OWN, LAST_OWN)
                           else torch.zeros(PLANE)) for c in (0, 1) for w in range(4)}
        counts = torch.tensor([rank + 1, 10 * (rank + 1)], dtype=torch.int64)
        halo = TorchHalo(lambda c, w: planes[(c, w)], counts, periodic)
        halo.exchange(1)
        halo.sum_counts(0)
        q.put((rank, {k: v.tolist() for k, v in planes.items()}, counts.tolist()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(120)
@pytest.mark.parametrize("world,periodic", [(2, True), (3, True), (3, False), (2, False)])
def test_halo_exchange_over_gloo(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, periodic, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        r, planes, counts = q.get(timeout=100)
        got[r] = (planes, counts)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    total = sum(r + 1 for r in range(world))
    for r in range(world):
        planes, counts = got[r]
        assert counts == [total, 10 * (r + 1)]  # only the director count was summed
        down = r - 1 if r > 0 else (world - 1 if periodic else None)
        up = r + 1 if r + 1 < world else (0 if periodic else None)
        lower = _pattern(down, 1, LAST_OWN).tolist() if down is not None else [0.0] * PLANE
        upper = _pattern(up, 1, FIRST_OWN).tolist() if up is not None else [0.0] * PLANE
        assert planes[(1, LOWER_HALO)] == lower
        assert planes[(1, UPPER_HALO)] == upper
        assert planes[(0, LOWER_HALO)] == [0.0] * PLANE  # colour 0 untouched
