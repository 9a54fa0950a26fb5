"""Workflow drivers built on the device lattice and the batch.

``anneal`` is the reference's temperature-annealing workflow
(scripts/pdanneal.py:18-37, scripts/pdlargeanneal1.0.py:36-53): there each
kT stage is a new process-level ChLLSim that reloads the previous stage's
NPZ; here the lattice stays on the GPU from stage to stage, the step
counter keeps running (so the Philox stream never repeats) and every stage
reports FP64 means and fluctuations.

``phase_diagram`` maps a (kT, g) grid as one batched launch instead of the
serial loops of scripts/phase_diagram.py:24-49 and scripts/g_field0.5.py:24-32.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .lattice import Lattice, coupling
from .observables import nematic_S


def linear_schedule(kT_start: float, kT_stop: float, stages: int) -> list[float]:
    return [float(x) for x in np.linspace(kT_start, kT_stop, stages)]


def anneal(lat: Lattice, schedule, sweeps_per_stage: int, *, K: float, g: float = 0.0,
           eps: float = 1.0, seed: int = 1, replica: int = 0, measure_every: int = 10,
           d0: float | None = None, step0: int = 1) -> list[dict]:
    """Sweeps `lat` through the kT schedule.  Returns one dict per stage with
    FP64 <e>, <eta>, <S>, C_v = N var(e)/kT^2, chi = N var(eta)/kT."""
    n = lat.nsites
    if d0 is not None:
        lat.set_control(d0, step=step0)
    per_stage = max(1, sweeps_per_stage // measure_every)
    lat.reserve_rows(per_stage)
    out = []
    for kT in schedule:
        cp = coupling(kT, K, g, eps)
        done = 0
        for r in range(per_stage):
            chunk = measure_every if r < per_stage - 1 else sweeps_per_stage - done
            lat.sweep(cp, chunk, seed=seed, replica=replica)
            done += chunk
            lat.measure(cp, r)
        rows = lat.read_rows(0, per_stage)
        e = rows[:, _lib.ROW_ENERGY] / n
        eta = rows[:, _lib.ROW_SUM_S] / n
        S = np.array([nematic_S(rw[_lib.ROW_QXX:_lib.ROW_QXX + 6], n) for rw in rows])
        ctl = lat.control()
        out.append({
            "kT": float(kT), "sweeps": done, "energy": float(e.mean()), "eta": float(eta.mean()),
            "abs_eta": float(np.abs(eta).mean()), "S": float(S.mean()),
            "C_v": float(n * e.var() / kT ** 2) if kT > 0 else float("nan"),
            "chi_c": float(n * eta.var() / kT) if kT > 0 else float("nan"),
            "d": ctl["d"], "step": ctl["step"], "paccept": ctl["paccept"],
        })
    return out


def phase_diagram(kTs, gs, sizes, *, K=1.0, eps=1.0, nsweeps=2000, measure_every=10,
                  measure_from=0, seed=1, autotune=True, init="random") -> list[dict]:
    """Every (kT, g) point as a replica of one batched launch; returns the
    per-replica FP64 summaries (energy, eta, S, C_v, chi_c).  init: "random"
    (directors uniform on the sphere), "aligned" (1,0,0), "aligned2"
    (1/sqrt2, 0, 1/sqrt2) as the reference drivers' init_aligned /
    init_aligned2, or any direction (x, y, z); spins are random either way."""
    from .batched import Batch, phase_grid

    specs = phase_grid(kTs, gs, sizes, K=K, eps=eps, seed=seed)
    directions = {"aligned": (1.0, 0.0, 0.0), "aligned2": (1.0, 0.0, 1.0)}
    with Batch(specs) as b:
        if isinstance(init, str) and init == "random":
            b.init_random()
        else:
            b.init_uniform(directions[init] if isinstance(init, str) else init)
        if autotune:
            b.autotune(trial_sweeps=10)
        b.run(nsweeps, measure_every, measure_from)
        return b.summary()
