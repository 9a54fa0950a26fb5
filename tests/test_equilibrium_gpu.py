"""Equilibrium parity: independent GPU and oracle chains at the same
couplings agree on <e>, <eta>, <S> and C_v = N var(e)/kT^2 within two
standard errors (batch means over 20 blocks; fixed seeds)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (8, 8, 8)
KT, K, H = 0.9, 1.0, 0.25
BURN, MEAS, EVERY = 2000, 16000, 8
NBLOCK = 20


def _stats(e, eta, S, n):
    def bm(x):
        b = np.asarray(x)[: len(x) // NBLOCK * NBLOCK].reshape(NBLOCK, -1).mean(1)
        return float(b.mean()), float(b.std(ddof=1) / math.sqrt(NBLOCK))

    blocks_e = np.asarray(e)[: len(e) // NBLOCK * NBLOCK].reshape(NBLOCK, -1)
    cv_blocks = n * blocks_e.var(axis=1) / KT ** 2
    cv = (float(cv_blocks.mean()), float(cv_blocks.std(ddof=1) / math.sqrt(NBLOCK)))
    return {"e": bm(e), "eta": bm(eta), "S": bm(S), "C_v": cv}


def test_equilibrium_averages_gpu_vs_oracle(oracle):
    from chllmodel_b200.lattice import Lattice, coupling
    from chllmodel_b200.observables import nematic_S

    n = int(np.prod(SHAPE))
    cp = coupling(KT, K, H)
    lat = Lattice(*SHAPE, boundary="periodic")
    lat.init_random(101)
    lat.set_control(0.1, step=1)
    lat.sweep(cp, BURN, seed=101)
    nm = MEAS // EVERY
    lat.reserve_rows(nm)
    for r in range(nm):
        lat.sweep(cp, EVERY, seed=101)
        lat.measure(cp, r)
    rows = lat.read_rows(0, nm)
    g = _stats(rows[:, 5] / n, rows[:, 6] / n,
               [nematic_S(r[7:13], n) for r in rows], n)
    lat.close()

    cfg = oracle.make_cfg(*SHAPE, periodic=True, kT=KT, K=K, g=H, seed=202)
    nx, ny, nz, s = oracle.init_random(oracle.make_cfg(*SHAPE, seed=202))
    oracle.set_threads(1)
    d = 0.1
    e, eta, S = [], [], []
    step = 1
    for sweep in range(BURN + MEAS):
        acc = 0
        for p in range(4):
            c = oracle.run_pass(cfg, p, step, d, nx, ny, nz, s)
            if p < 2:
                acc += c
        pa = float(np.float32(acc) / np.float32(n))
        if step < 10000:
            f = float(np.float32(0.995))
            d = d * f if pa < 0.4 else (d / f if pa > 0.6 else d)
        step += 1
        if sweep >= BURN and (sweep - BURN + 1) % EVERY == 0:
            mo = oracle.moments(cfg, nx, ny, nz, s)
            e.append(mo[0] / n)
            eta.append(mo[2] / n)
            S.append(nematic_S(mo[3:9], n))
    o = _stats(e, eta, S, n)
    for key in ("e", "eta", "S", "C_v"):
        (mg, sg), (mo_, so) = g[key], o[key]
        se = math.sqrt(sg * sg + so * so)
        assert abs(mg - mo_) <= 2 * se + 1e-12, f"{key}: gpu {mg}+-{sg} oracle {mo_}+-{so}"
