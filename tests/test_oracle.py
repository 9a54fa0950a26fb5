"""CPU tests of the oracle: pinned against the reference's own golden data
(the notebook ekernel fixture, the published Philox vectors, the analytic
K=0 limit the reference notebooks check) and against independent numpy
restatements of chll_mod.f90's energy and etot."""
import json
import math
import os

import numpy as np
import pytest


def rand_state(shape, seed):
    rng = np.random.default_rng(seed)
    ct = rng.uniform(-1, 1, shape)
    st = np.sqrt(1 - ct * ct)
    ph = rng.uniform(0, 2 * np.pi, shape)
    f = lambda a: np.asfortranarray(a)
    s = np.where(rng.random(shape) < 0.5, -1, 1).astype(np.int32)
    return f(st * np.cos(ph)), f(st * np.sin(ph)), f(ct), np.asfortranarray(s)


def np_site_energy(nx, ny, nz, s, i, j, k, m, snew, K, g, eps=1.0, periodic=False):
    """Independent FP64 restatement of chll_mod.f90:363-412 (no FP32 rounding)."""
    ni, nj, nk = nx.shape
    e = 0.0
    n = np.array(m, dtype=np.float64)
    for axis, (sh, size) in enumerate([((1, 0, 0), ni), ((0, 1, 0), nj), ((0, 0, 1), nk)]):
        for sgn in (+1, -1):
            q = np.array([i, j, k]) + sgn * np.array(sh)
            if q[axis] < 0 or q[axis] >= size:
                if not periodic:
                    continue
                q[axis] %= size
            b = np.array([nx[tuple(q)], ny[tuple(q)], nz[tuple(q)]])
            dot = n @ b
            cr = np.cross(n, b)[axis]
            sfac = 0.5 * (snew + s[tuple(q)])
            e += eps * (1 - dot * dot) - sgn * K * dot * cr * sfac
    return e - g * snew


def np_etot_reference(nx, ny, nz, s, K, g):
    """Independent restatement of etot (chll_mod.f90:414-456), incl. the +y typo."""
    ni, nj, nk = nx.shape
    e = 0.0
    for k in range(nk):
        for j in range(nj):
            for i in range(ni):
                ip, jp = (i + 1) % ni, (j + 1) % nj
                d = nx[i, j, k] * nx[ip, j, k] + ny[i, j, k] * ny[ip, j, k] + nz[i, j, k] * nz[ip, j, k]
                c = ny[i, j, k] * nz[ip, j, k] - nz[i, j, k] * ny[ip, j, k]
                e += (1 - d * d) - K * d * c * 0.5 * (s[i, j, k] + s[ip, j, k])
                d = nx[i, j, k] * nx[ip, jp, k] + ny[i, j, k] * ny[i, jp, k] + nz[i, j, k] * nz[i, jp, k]
                c = nz[i, j, k] * nx[i, jp, k] - nx[i, j, k] * nz[i, jp, k]
                e += (1 - d * d) - K * d * c * 0.5 * (s[i, j, k] + s[i, jp, k])
                if k + 1 < nk:
                    d = nx[i, j, k] * nx[i, j, k + 1] + ny[i, j, k] * ny[i, j, k + 1] + nz[i, j, k] * nz[i, j, k + 1]
                    c = nx[i, j, k] * ny[i, j, k + 1] - ny[i, j, k] * nx[i, j, k + 1]
                    e += (1 - d * d) - K * d * c * 0.5 * (s[i, j, k] + s[i, j, k + 1])
                e -= g * s[i, j, k]
    return e


def test_philox_known_answers(oracle, golden_dir):
    kat = json.load(open(os.path.join(golden_dir, "philox_kat.json")))
    for ctr, key, out in kat["vectors"]:
        assert oracle.philox(ctr, key) == out


def test_oracle_energy_matches_reference_ekernel(oracle, golden_dir):
    """The notebook's ekernel (KK=1, no field) on interior sites."""
    d = np.load(os.path.join(golden_dir, "ekernel_energy.npz"))
    checked = 0
    for c in range(int(d["ncases"])):
        nx, ny, nz = (np.asfortranarray(d[f"c{c}_{a}"]) for a in ("nx", "ny", "nz"))
        s = np.asfortranarray(d[f"c{c}_s"]).astype(np.int32)
        e = d[f"c{c}_e"]
        ni, nj, nk = nx.shape
        cfg = oracle.make_cfg(ni, nj, nk, K=float(d["KK"]), g=0.0)
        for i, j, k in zip(*np.nonzero(~np.isnan(e))):
            v = oracle.site_energy(cfg, nx, ny, nz, s, int(i), int(j), int(k))
            # oracle accumulates in FP32 like the Fortran energy() result
            assert v == pytest.approx(e[i, j, k], rel=2e-6, abs=2e-6)
            checked += 1
    assert checked > 50


@pytest.mark.parametrize("periodic", [False, True])
def test_oracle_energy_matches_numpy_restatement(oracle, periodic):
    shape = (6, 4, 8)
    nx, ny, nz, s = rand_state(shape, 3)
    cfg = oracle.make_cfg(*shape, periodic=periodic, K=0.7, g=0.3, eps=1.3)
    rng = np.random.default_rng(5)
    for _ in range(60):
        i, j, k = (int(rng.integers(0, n)) for n in shape)
        m = rng.normal(size=3)
        m /= np.linalg.norm(m)
        for snew in (-1, 1):
            ref = np_site_energy(nx, ny, nz, s, i, j, k, m, snew, 0.7, 0.3, 1.3, periodic)
            got = oracle.site_energy(cfg, nx, ny, nz, s, i, j, k, m, snew)
            assert got == pytest.approx(ref, rel=3e-6, abs=3e-6)


def test_oracle_etot_reference_quirks(oracle):
    shape = (5, 4, 3)
    nx, ny, nz, s = rand_state(shape, 11)
    cfg = oracle.make_cfg(*shape, K=0.9, g=0.2)
    v32, tot = oracle.etot(cfg, nx, ny, nz, s, mode=0)
    ref = np_etot_reference(nx, ny, nz, s, 0.9, 0.2)
    assert tot == pytest.approx(ref, rel=1e-12)
    assert v32 == np.float32(ref / np.float32(np.prod(shape)))


@pytest.mark.parametrize("periodic", [False, True])
def test_local_energy_difference_equals_total(oracle, periodic):
    """Changing one site changes the consistent total energy by exactly its
    local energy difference (the sweep's dE and the observable agree)."""
    shape = (6, 6, 4)
    nx, ny, nz, s = rand_state(shape, 7)
    cfg = oracle.make_cfg(*shape, periodic=periodic, K=1.1, g=0.4, eps=0.8)
    for (i, j, k) in [(0, 0, 0), (5, 5, 3), (2, 3, 1), (0, 5, 2)]:
        _, e0 = oracle.etot(cfg, nx, ny, nz, s, mode=1)
        loc0 = np_site_energy(nx, ny, nz, s, i, j, k, (nx[i, j, k], ny[i, j, k], nz[i, j, k]),
                              s[i, j, k], 1.1, 0.4, 0.8, periodic)
        old = (nx[i, j, k], ny[i, j, k], nz[i, j, k], s[i, j, k])
        m = np.array([0.3, -0.5, 0.81])
        m /= np.linalg.norm(m)
        nx[i, j, k], ny[i, j, k], nz[i, j, k] = m
        s[i, j, k] = -s[i, j, k]
        _, e1 = oracle.etot(cfg, nx, ny, nz, s, mode=1)
        loc1 = np_site_energy(nx, ny, nz, s, i, j, k, m, s[i, j, k], 1.1, 0.4, 0.8, periodic)
        assert e1 - e0 == pytest.approx(loc1 - loc0, rel=1e-10, abs=1e-10)
        nx[i, j, k], ny[i, j, k], nz[i, j, k], s[i, j, k] = old


def test_oracle_pass_rule(oracle):
    """Per-site decisions follow chll_mod.f90:188-200; other colour untouched."""
    shape = (8, 6, 4)
    nx, ny, nz, s = rand_state(shape, 1)
    cfg = oracle.make_cfg(*shape, kT=0.4, K=0.5, g=0.1)
    for p in range(4):
        before = [a.copy() for a in (nx, ny, nz, s)]
        n, acc, de, u = oracle.run_pass(cfg, p, 17, 0.2, nx, ny, nz, s, detail=True)
        i, j, k = np.indices(shape)
        mine = ((i + j + k) & 1) == (p & 1)
        assert np.all(acc[mine] >= 0) and np.all(acc[~mine] == -1)
        exp_acc = (de < 0) | (u <= np.exp(-de / 0.4))
        assert np.array_equal(acc[mine] == 1, exp_acc[mine])
        assert n == int((acc == 1).sum())
        for a, b in zip((nx, ny, nz, s), before):
            assert np.array_equal(a[~mine], b[~mine])
        if p >= 2:
            flipped = s != before[3]
            assert np.array_equal(flipped, acc == 1)


def test_oracle_director_proposal_is_tangent_rotation(oracle):
    rng = np.random.default_rng(2)
    for _ in range(200):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        d, u = 0.1, rng.random()
        m = oracle.propose(n, d, u)
        assert np.linalg.norm(m) == pytest.approx(1.0, abs=1e-14)
        if abs(n[2]) <= 0.999:
            # |m - n| equals the chord of a tangent step of length d
            assert np.linalg.norm(m * np.sqrt(1 + d * d) - n) == pytest.approx(d, rel=1e-9)


def test_oracle_run_rows_and_d_adaptation(oracle):
    shape = (8, 8, 8)
    cfg = oracle.make_cfg(*shape, kT=0.5, K=0.5, seed=9)
    nx, ny, nz, s = oracle.init_random(cfg)
    msteps, m, d, nmeas = oracle.run(cfg, 1, 120, 40, 0.1, nx, ny, nz, s)
    assert list(msteps) == [40, 80, 120] and nmeas == 3
    # paccept/faccept are FP32 fractions of N; d is the adapted value
    for r in range(3):
        assert 0.0 <= m[r, 2] <= 1.0 and 0.0 <= m[r, 3] <= 1.0
        assert m[r, 2] * 512 == pytest.approx(round(m[r, 2] * 512), abs=1e-3)
    assert m[2, 4] == d
    # d only moves in factors of the FP32 literal 0.995
    ratio = math.log(d / 0.1) / math.log(float(np.float32(0.995)))
    assert ratio == pytest.approx(round(ratio), abs=1e-6)
    # the last row's etot and eta are those of the final state
    v32, _ = oracle.etot(cfg, nx, ny, nz, s, mode=0)
    assert m[2, 0] == v32
    assert m[2, 1] == np.float32(np.float32(s.sum()) / np.float32(512))


def test_oracle_zero_temperature(oracle):
    """kT = 0: only downhill moves (and u == 0) are accepted, as the
    reference's exp(-dE/0) gives."""
    shape = (6, 6, 6)
    cfg = oracle.make_cfg(*shape, kT=0.0, K=1.0, g=0.5, seed=4)
    nx, ny, nz, s = oracle.init_random(cfg)
    for p in range(4):
        n, acc, de, u = oracle.run_pass(cfg, p, 3, 0.1, nx, ny, nz, s, detail=True)
        mask = acc >= 0
        assert np.all((acc[mask] == 1) == ((de[mask] < 0) | ((de[mask] > 0) & (u[mask] == 0))))


def test_oracle_k0_field_limit(oracle):
    """With K = 0 the chiralities are independent spins in field g, so
    <s> = tanh(g/kT): the known-answer check of the reference notebooks
    (paper_plots2.ipynb cells 3-4)."""
    shape = (8, 8, 8)
    kT, g = 0.5, 0.2
    cfg = oracle.make_cfg(*shape, kT=kT, K=0.0, g=g, seed=21)
    nx, ny, nz, s = oracle.init_random(cfg)
    vals = []
    for step in range(1, 1201):
        for p in (2, 3):
            oracle.run_pass(cfg, p, step, 0.1, nx, ny, nz, s)
        if step > 200:
            vals.append(s.mean())
    vals = np.array(vals)
    nb = 20
    bm = vals[: len(vals) // nb * nb].reshape(nb, -1).mean(axis=1)
    se = bm.std(ddof=1) / math.sqrt(nb)
    assert abs(vals.mean() - math.tanh(g / kT)) < 3 * se + 1e-3


def test_oracle_gradient_central_differences(oracle):
    shape = (5, 4, 6)
    nx, ny, nz, s = rand_state(shape, 8)
    for periodic in (False, True):
        if periodic:
            shape2 = (4, 4, 6)
            nx, ny, nz, s = rand_state(shape2, 8)
        sh = nx.shape
        cfg = oracle.make_cfg(*sh, periodic=periodic, K=0.8, g=0.3, eps=1.2)
        grad, out4 = oracle.energy_grad(cfg, nx, ny, nz, s)
        _, e_tot = oracle.etot(cfg, nx, ny, nz, s, mode=1)
        assert out4[0] == pytest.approx(e_tot, rel=1e-12)
        h = 1e-5
        rng = np.random.default_rng(1)
        for _ in range(20):
            x = tuple(int(rng.integers(0, n)) for n in sh)
            for comp, arr in enumerate((nx, ny, nz)):
                old = arr[x]
                arr[x] = old + h
                ep = oracle.etot(cfg, nx, ny, nz, s, mode=1)[1]
                arr[x] = old - h
                em = oracle.etot(cfg, nx, ny, nz, s, mode=1)[1]
                arr[x] = old
                assert grad[x + (comp,)] == pytest.approx((ep - em) / (2 * h), abs=1e-6)
        # coupling derivatives
        for name, idx in (("eps", 1), ("K", 2), ("g", 3)):
            c2 = oracle.make_cfg(*sh, periodic=periodic, K=0.8, g=0.3, eps=1.2)
            cm = oracle.make_cfg(*sh, periodic=periodic, K=0.8, g=0.3, eps=1.2)
            setattr(c2, name, getattr(c2, name) + h)
            setattr(cm, name, getattr(cm, name) - h)
            fd = (oracle.etot(c2, nx, ny, nz, s, 1)[1] - oracle.etot(cm, nx, ny, nz, s, 1)[1]) / (2 * h)
            assert out4[idx] == pytest.approx(fd, rel=1e-6, abs=1e-6)
