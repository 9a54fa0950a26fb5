"""Replica sharding across GPUs (one process per GPU, torch.distributed).

Independent replicas (phase-diagram points, seeds) need no exchange while
they run, so a grid is split across ranks by work (sites x sweeps, longest
first onto the least-loaded rank), each rank sweeps its share as one batched
launch on its own GPU, and the per-replica FP64 summaries are gathered once
at the end.  There is no collective on the data path.
"""
from __future__ import annotations

from typing import Callable, Sequence


def shard(specs: Sequence[dict], world: int) -> list[list[int]]:
    """Replica indices per rank, balancing sites (longest-processing-time
    first).  Deterministic for a given spec list and world size."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(specs)),
                   key=lambda i: (-specs[i]["ni"] * specs[i]["nj"] * specs[i]["nk"], i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += specs[i]["ni"] * specs[i]["nj"] * specs[i]["nk"]
    return [sorted(p) for p in parts]


def run_sharded(specs: Sequence[dict], runner: Callable[[list[dict]], list[dict]],
                rank: int, world: int, gather: Callable | None = None) -> list[dict] | None:
    """Runs this rank's share with `runner` (a list of specs -> a list of
    per-replica results) and gathers all results, in spec order, to rank 0
    (other ranks get None).  `gather` defaults to torch.distributed's
    gather_object on an initialised process group."""
    parts = shard(specs, world)
    mine = parts[rank]
    results = runner([specs[i] for i in mine]) if mine else []
    tagged = list(zip(mine, results))
    if world == 1:
        collected = [tagged]
    else:
        if gather is None:
            import torch.distributed as dist

            collected = [None] * world if rank == 0 else None
            dist.gather_object(tagged, collected, dst=0)
        else:
            collected = gather(tagged)
    if rank != 0:
        return None
    out: list = [None] * len(specs)
    for part in collected:
        for i, res in part:
            out[i] = res
    return out


def batch_runner(nsweeps: int, measure_every: int = 10, measure_from: int = 0,
                 autotune: bool = True) -> Callable[[list[dict]], list[dict]]:
    """Runner for run_sharded that sweeps a share as one Batch on the
    current CUDA device."""

    def _run(share: list[dict]) -> list[dict]:
        from .batched import Batch

        with Batch(share) as b:
            b.init_random()
            if autotune:
                b.autotune(trial_sweeps=10)
            b.run(nsweeps, measure_every, measure_from)
            return b.summary()

    return _run
