"""Equilibrium parity: independent GPU and oracle chains at the same
couplings agree on <e>, <eta>, <S>, C_v = N var(e)/kT^2 and the chiral
susceptibility chi_c = N var(eta)/kT within two standard errors.

Each side runs NCHAIN independent chains (own seeds and initial states), and
each chain gives one estimate of every quantity; the standard error of a
side is the spread of its chain estimates over sqrt(NCHAIN).  Estimates from
independent chains carry no autocorrelation, which a single chain's batch
means underestimate here (two long oracle chains at the anneal-stage
couplings disagreed by 2.8 batch-means errors on <e>).

Cases: a reference point (kT 0.9, K 1, h 0.25); the couplings of the 32^3
reference-size run (kT 0.5, K 0.5, h 0); and stage 4 of the 128^3 anneal
(K 1, h 0.25, kT on linspace(1.5, 0.1, 20): the isotropic side, where the
chain mixes).  chi_c is the variance of notebooks/.ipynb_checkpoints/
Xch-checkpoint.ipynb cell 2 times N/kT, as paper_plots-checkpoint cell 8."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NCHAIN = 10
BURN, NMEAS, EVERY = 2000, 1000, 8
ANNEAL_KT = [float(x) for x in np.linspace(1.5, 0.1, 20)]
KEYS = ("e", "eta", "S", "C_v", "chi_c")

CASES = [
    # name, shape, kT, K, h
    ("reference_point", (8, 8, 8), 0.9, 1.0, 0.25),
    ("plain_32_couplings", (12, 12, 12), 0.5, 0.5, 0.0),
    ("anneal_128_stage4", (12, 12, 12), ANNEAL_KT[4], 1.0, 0.25),
]


def _chain_estimates(mom, n, kT):
    """One chain's estimates from its FP64 moment rows (E, sum s, Q sums)."""
    from chllmodel_b200.observables import nematic_S

    e = mom[:, 0] / n
    eta = mom[:, 1] / n
    S = np.array([nematic_S(q, n) for q in mom[:, 2:8]])
    return {"e": e.mean(), "eta": eta.mean(), "S": S.mean(), "C_v": n * e.var() / kT ** 2,
            "chi_c": n * eta.var() / kT}


def _gpu_chains(shape, kT, K, h):
    from chllmodel_b200.lattice import Lattice, coupling

    n = int(np.prod(shape))
    cp = coupling(kT, K, h)
    out = []
    for c in range(NCHAIN):
        seed = 1001 + 7 * c
        lat = Lattice(*shape, boundary="periodic")
        lat.init_random(seed)
        lat.set_control(0.1, step=1)
        lat.sweep(cp, BURN, seed=seed)
        lat.reserve_rows(NMEAS)
        for r in range(NMEAS):
            lat.sweep(cp, EVERY, seed=seed)
            lat.measure(cp, r)
        rows = lat.read_rows(0, NMEAS)
        lat.close()
        out.append(_chain_estimates(np.column_stack([rows[:, 5], rows[:, 6], rows[:, 7:13]]),
                                    n, kT))
    return out


def _oracle_chains(oracle, shape, kT, K, h):
    n = int(np.prod(shape))
    out = []
    for c in range(NCHAIN):
        seed = 5003 + 7 * c
        cfg = oracle.make_cfg(*shape, periodic=True, kT=kT, K=K, g=h, seed=seed)
        nx, ny, nz, s = oracle.init_random(oracle.make_cfg(*shape, seed=seed))
        mom, _ = oracle.chain(cfg, BURN, NMEAS, EVERY, 0.1, nx, ny, nz, s)
        out.append(_chain_estimates(np.column_stack([mom[:, 0], mom[:, 2:9]]), n, kT))
    return out


def _mean_se(chains, key):
    x = np.array([c[key] for c in chains])
    return float(x.mean()), float(x.std(ddof=1) / math.sqrt(len(x)))


@pytest.mark.parametrize("name,shape,kT,K,h", CASES, ids=[c[0] for c in CASES])
def test_equilibrium_averages_gpu_vs_oracle(oracle, name, shape, kT, K, h):
    oracle.set_threads(oracle.max_threads())
    g = _gpu_chains(shape, kT, K, h)
    o = _oracle_chains(oracle, shape, kT, K, h)
    for key in KEYS:
        (mg, sg), (mo, so) = _mean_se(g, key), _mean_se(o, key)
        se = math.sqrt(sg * sg + so * so)
        assert abs(mg - mo) <= 2 * se + 1e-12, f"{name} {key}: gpu {mg}+-{sg} oracle {mo}+-{so}"
