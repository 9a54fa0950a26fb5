"""Equilibrium parity: independent GPU and oracle chains at the same
couplings agree on <e>, <eta>, <S>, C_v = N var(e)/kT^2 and the chiral
susceptibility chi_c = N var(eta)/kT within two standard errors (batch means
over 20 blocks; fixed seeds).

Cases: a reference point (kT 0.9, K 1, h 0.25); the couplings of the 32^3
reference-size run (kT 0.5, K 0.5, h 0); and stage 4 of the 128^3 anneal
(K 1, h 0.25, kT on linspace(1.5, 0.1, 20): the isotropic side, where the
chain mixes).  chi_c is the variance of notebooks/.ipynb_checkpoints/
Xch-checkpoint.ipynb cell 2 times N/kT, as paper_plots-checkpoint cell 8."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BURN, MEAS, EVERY = 2000, 16000, 8
NBLOCK = 20
ANNEAL_KT = [float(x) for x in np.linspace(1.5, 0.1, 20)]

CASES = [
    # name, shape, kT, K, h
    ("reference_point", (8, 8, 8), 0.9, 1.0, 0.25),
    ("plain_32_couplings", (12, 12, 12), 0.5, 0.5, 0.0),
    ("anneal_128_stage4", (12, 12, 12), ANNEAL_KT[4], 1.0, 0.25),
]


def _stats(e, eta, S, n, kT):
    def blocks(x):
        return np.asarray(x)[: len(x) // NBLOCK * NBLOCK].reshape(NBLOCK, -1)

    def mean_se(b):
        return float(b.mean()), float(b.std(ddof=1) / math.sqrt(NBLOCK))

    cv_blocks = n * blocks(e).var(axis=1) / kT ** 2
    chi_blocks = n * blocks(eta).var(axis=1) / kT
    return {"e": mean_se(blocks(e).mean(1)), "eta": mean_se(blocks(eta).mean(1)),
            "S": mean_se(blocks(S).mean(1)), "C_v": mean_se(cv_blocks),
            "chi_c": mean_se(chi_blocks)}


def _gpu_chain(shape, kT, K, h):
    from chllmodel_b200.lattice import Lattice, coupling
    from chllmodel_b200.observables import nematic_S

    n = int(np.prod(shape))
    cp = coupling(kT, K, h)
    lat = Lattice(*shape, boundary="periodic")
    lat.init_random(101)
    lat.set_control(0.1, step=1)
    lat.sweep(cp, BURN, seed=101)
    nm = MEAS // EVERY
    lat.reserve_rows(nm)
    for r in range(nm):
        lat.sweep(cp, EVERY, seed=101)
        lat.measure(cp, r)
    rows = lat.read_rows(0, nm)
    lat.close()
    return _stats(rows[:, 5] / n, rows[:, 6] / n, [nematic_S(r[7:13], n) for r in rows], n, kT)


def _oracle_chain(oracle, shape, kT, K, h):
    from chllmodel_b200.observables import nematic_S

    n = int(np.prod(shape))
    cfg = oracle.make_cfg(*shape, periodic=True, kT=kT, K=K, g=h, seed=202)
    nx, ny, nz, s = oracle.init_random(oracle.make_cfg(*shape, seed=202))
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
        # the reference's step-size rule (chll_mod.f90:83-90)
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
    return _stats(e, eta, S, n, kT)


@pytest.mark.parametrize("name,shape,kT,K,h", CASES, ids=[c[0] for c in CASES])
def test_equilibrium_averages_gpu_vs_oracle(oracle, name, shape, kT, K, h):
    g = _gpu_chain(shape, kT, K, h)
    o = _oracle_chain(oracle, shape, kT, K, h)
    for key in ("e", "eta", "S", "C_v", "chi_c"):
        (mg, sg), (mo_, so) = g[key], o[key]
        se = math.sqrt(sg * sg + so * so)
        assert abs(mg - mo_) <= 2 * se + 1e-12, f"{name} {key}: gpu {mg}+-{sg} oracle {mo_}+-{so}"
