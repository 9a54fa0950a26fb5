"""Batched replicas: a whole phase-diagram grid in one persistent launch.

The reference maps a (kT, K, g) grid with one process and one ``ChLLSim`` per
point, run one after another (scripts/phase_diagram.py:24-31,
scripts/g_field0.5.py:24-31, scripts/pdanneal.py:18-37).  ``Batch`` holds
every point as a replica of its own size and couplings on one GPU, sweeps all
of them in one cooperative persistent kernel (captured as a CUDA graph) and
accumulates FP64 energy, chirality, nematic order and their fluctuations per
replica on the device.  ``autotune`` picks the launch shape (threads per CTA
and CTAs per SM) by timing trial sweeps on the actual replica set.
"""
from __future__ import annotations

import ctypes as ct
import json
import os

import numpy as np

from . import _lib
from ._lib import ReplicaSpec, check
from .observables import summarize_batch


def replica(ni, nj=None, nk=None, *, kT, K, g=0.0, eps=1.0, d=0.1, seed=1, replica=0,
            boundary="periodic") -> dict:
    nj = ni if nj is None else nj
    nk = ni if nk is None else nk
    return {"ni": int(ni), "nj": int(nj), "nk": int(nk), "kT": float(kT), "K": float(K),
            "g": float(g), "eps": float(eps), "d": float(d), "seed": int(seed),
            "replica": int(replica), "boundary": boundary}


def phase_grid(kTs, gs, sizes, *, K=1.0, eps=1.0, d=0.1, seed=1, size_seed=None,
               boundary="periodic") -> list[dict]:
    """One replica per (kT, g) pair, lattice edge drawn uniformly from `sizes`
    (seeded by size_seed, default seed), replica i seeded `seed + i`."""
    rng = np.random.default_rng(seed if size_seed is None else size_seed)
    specs = []
    for kT in kTs:
        for g in gs:
            i = len(specs)
            L = int(rng.choice(np.asarray(sizes)))
            specs.append(replica(L, kT=kT, K=K, g=g, eps=eps, d=d, seed=seed + i, replica=i,
                                 boundary=boundary))
    return specs


def _spec_struct(sp: dict) -> ReplicaSpec:
    return ReplicaSpec(sp["ni"], sp["nj"], sp["nk"],
                       _lib.CHLL_PERIODIC if sp["boundary"] == "periodic" else _lib.CHLL_OPEN,
                       sp["kT"], sp["K"], sp["g"], sp["eps"], sp["d"], sp["seed"],
                       sp["replica"], 0)


class Batch:
    def __init__(self, specs: list[dict]):
        self._L = _lib.load()
        self.specs = [dict(s) for s in specs]
        arr = (ReplicaSpec * len(specs))(*[_spec_struct(s) for s in specs])
        h = ct.c_void_p()
        check(self._L.chll_batch_create(arr, len(specs), ct.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.chll_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self.specs)

    def set_stream(self, stream_ptr):
        check(self._L.chll_batch_set_stream(self._h, ct.c_void_p(stream_ptr or 0)))

    def sync(self):
        check(self._L.chll_batch_sync(self._h))

    def init_random(self):
        check(self._L.chll_batch_init_random(self._h))

    def init_uniform(self, direction, spin_seed=None):
        """Every site of every replica gets the director `direction` (normalised;
        the reference drivers' init_aligned (1,0,0) and init_aligned2
        (1/sqrt2, 0, 1/sqrt2), e.g. scripts/phase_diagram_large_lowT_1.0.py:18-26)
        and a chirality of -1 or +1 with probability 1/2 each (as init_rand_s),
        drawn from numpy's generator seeded with (spin_seed or the replica's
        seed, replica index)."""
        v = np.asarray(direction, np.float64)
        v = (v / np.linalg.norm(v)).astype(np.float32)
        for r, sp in enumerate(self.specs):
            n = sp["ni"] * sp["nj"] * sp["nk"]
            rng = np.random.default_rng([sp["seed"] if spin_seed is None else int(spin_seed), r])
            f4 = np.empty((n, 4), np.float32)
            f4[:, :3] = v
            f4[:, 3] = np.where(rng.random(n) < 0.5, -1.0, 1.0)
            self.upload_f4(r, f4)

    def upload_f4(self, r, xyzs):
        a = np.ascontiguousarray(xyzs, dtype=np.float32)
        check(self._L.chll_batch_upload_f4(self._h, int(r), a.ctypes.data_as(ct.c_void_p)))

    def download_f4(self, r):
        sp = self.specs[r]
        a = np.zeros((sp["ni"] * sp["nj"] * sp["nk"], 4), np.float32)
        check(self._L.chll_batch_download_f4(self._h, int(r), a.ctypes.data_as(ct.c_void_p)))
        return a

    def run(self, nsweeps, measure_every=10, measure_from=0):
        """Enqueues nsweeps sweeps of every replica (asynchronous)."""
        check(self._L.chll_batch_run(self._h, int(nsweeps), int(measure_every),
                                     int(measure_from)))

    def moments(self) -> np.ndarray:
        m = np.zeros((len(self.specs), 16), np.float64)
        check(self._L.chll_batch_moments(self._h, m.ctypes.data_as(ct.c_void_p)))
        return m

    def summary(self) -> list[dict]:
        return summarize_batch(self.moments(), self.specs)

    def info(self) -> dict:
        n, r, t, g = ct.c_int64(), ct.c_int32(), ct.c_int32(), ct.c_int32()
        check(self._L.chll_batch_info(self._h, ct.byref(n), ct.byref(r), ct.byref(t),
                                      ct.byref(g)))
        return {"total_sites": n.value, "replicas": r.value, "threads": t.value, "grid": g.value}

    def set_tuning(self, threads, ctas_per_sm=0, wave_bytes=None, paired=None, pooled=None):
        """Launch shape (threads per CTA, CTAs per SM; 0: all that fit), wave
        size in bytes of state (0: one wave) and whether replica groups hold
        two replicas that alternate their passes or one (the default) -- all
        for the persistent launch -- and whether to sweep as pooled passes
        instead (one launch per pass over all replicas)."""
        check(self._L.chll_batch_set_tuning(self._h, int(threads), int(ctas_per_sm)))
        if wave_bytes is not None:
            check(self._L.chll_batch_set_wave_bytes(self._h, int(wave_bytes)))
        if paired is not None:
            check(self._L.chll_batch_set_pairing(self._h, int(bool(paired))))
        if pooled is not None:
            check(self._L.chll_batch_set_pooled(self._h, int(bool(pooled))))

    def set_wait_limit(self, polls):
        """Polls a replica group's barrier wait makes before it gives up and
        sets the replica's status word (default 2^24)."""
        check(self._L.chll_batch_set_wait_limit(self._h, int(polls)))

    def tuning(self) -> dict:
        t, c, w, n, p = ct.c_int32(), ct.c_int32(), ct.c_int64(), ct.c_int32(), ct.c_int32()
        check(self._L.chll_batch_get_tuning(self._h, ct.byref(t), ct.byref(c), ct.byref(w),
                                            ct.byref(n)))
        check(self._L.chll_batch_get_pairing(self._h, ct.byref(p)))
        q = ct.c_int32()
        check(self._L.chll_batch_get_pooled(self._h, ct.byref(q)))
        return {"threads": t.value, "ctas_per_sm": c.value, "wave_bytes": w.value,
                "waves": n.value, "paired": bool(p.value), "pooled": bool(q.value)}

    def autotune(self, trial_sweeps=20, cache=None) -> dict:
        """Times every launch shape on this replica set and keeps the fastest.
        With `cache` (a JSON path) the choice is stored per GPU and size mix."""
        key = self._tune_key()
        if cache and os.path.exists(cache):
            with open(cache) as f:
                table = json.load(f)
            if key in table:
                e = table[key]
                self.set_tuning(e["threads"], e["ctas_per_sm"], e.get("wave_bytes"),
                                e.get("paired"), e.get("pooled"))
                return dict(e, cached=True)
        t, c, ms = ct.c_int(), ct.c_int(), ct.c_double()
        check(self._L.chll_batch_autotune(self._h, int(trial_sweeps), ct.byref(t), ct.byref(c),
                                          ct.byref(ms)))
        tun = self.tuning()
        res = {"threads": t.value, "ctas_per_sm": c.value, "wave_bytes": tun["wave_bytes"],
               "waves": tun["waves"], "paired": tun["paired"], "pooled": tun["pooled"],
               "trial_ms": ms.value,
               "trial_sweeps": int(trial_sweeps)}
        if cache:
            table = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    table = json.load(f)
            table[key] = res
            with open(cache, "w") as f:
                json.dump(table, f, indent=1)
        return dict(res, cached=False)

    def _tune_key(self) -> str:
        try:
            import torch

            name = torch.cuda.get_device_name()
        except Exception:  # noqa: BLE001
            name = "cuda"
        sizes = sorted({(s["ni"], s["nj"], s["nk"]) for s in self.specs})
        hist = {str(sz): sum(1 for s in self.specs if (s["ni"], s["nj"], s["nk"]) == sz)
                for sz in sizes}
        return f"{name}|{json.dumps(hist, sort_keys=True)}"
