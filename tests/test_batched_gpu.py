"""GPU tests of the batched persistent launch.

Each replica of a batch shares the plain kernel's per-unit code and random
stream, so its chain must equal the same lattice run alone bit for bit, and
its FP64 measurements must equal the plain observables of its final state.
The K = 0 limit <s> = tanh(g/kT) (the reference notebooks' known answer) is
checked across a field grid in one launch."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _specs():
    from chllmodel_b200.batched import replica

    return [
        replica(16, kT=0.5, K=1.0, g=0.25, seed=3, replica=0),
        replica(8, 12, 6, kT=1.2, K=0.5, g=0.0, seed=4, replica=1),
        replica(12, kT=0.3, K=1.0, g=0.5, eps=1.3, d=0.2, seed=5, replica=2),
        replica(7, 5, 9, kT=0.8, K=0.7, g=0.1, seed=6, replica=3, boundary="open"),
        replica(24, 16, 20, kT=0.1, K=1.0, g=0.0, seed=7, replica=4),
    ]


@pytest.mark.parametrize("threads,wave_bytes,paired,pooled",
                         [(128, 0, True, False), (128, 0, False, False), (256, 1, True, False),
                          (512, 48 << 20, True, False), (128, 64 << 10, True, False),
                          (256, 64 << 10, False, False), (256, 0, False, True)])
def test_batch_replicas_equal_plain_runs(threads, wave_bytes, paired, pooled):
    """Any launch shape, wave split and grouping (two replicas alternating
    their passes, or one) of the persistent launch, and the pooled passes,
    give every replica its plain chain."""
    from chllmodel_b200.batched import Batch
    from chllmodel_b200.lattice import Lattice, coupling

    specs = _specs()
    nsw = 13
    with Batch(specs) as b:
        b.set_tuning(threads, 0, wave_bytes, paired, pooled)
        assert b.tuning()["paired"] == paired and b.tuning()["pooled"] == pooled
        if wave_bytes == 1:
            assert b.tuning()["waves"] == len(specs)  # every replica its own wave
        if wave_bytes == 64 << 10:
            assert b.tuning()["waves"] == 3  # 123 KB | 64 KB | 27 + 9 + 6 KB
        b.init_random()
        b.run(nsw, measure_every=4, measure_from=0)
        mom = b.moments()
        states = [b.download_f4(r) for r in range(len(specs))]
    for r, sp in enumerate(specs):
        lat = Lattice(sp["ni"], sp["nj"], sp["nk"], boundary=sp["boundary"])
        lat.init_random(sp["seed"], sp["replica"])
        lat.set_control(sp["d"], step=1, adapt_until=10000)
        cp = coupling(sp["kT"], sp["K"], sp["g"], sp["eps"])
        lat.sweep(cp, nsw, seed=sp["seed"], replica=sp["replica"])
        assert np.array_equal(lat.download_f4(), states[r]), f"replica {r} state differs"
        ctl = lat.control()
        assert mom[r, 11] == ctl["d"] and int(mom[r, 12]) == ctl["step"] == nsw + 1
        assert mom[r, 13] == ctl["paccept"] and mom[r, 14] == ctl["faccept"]
        # last measurement (after sweep 12) is not the final state; check count
        assert int(mom[r, 0]) == nsw // 4
        lat.close()


@pytest.mark.parametrize("pooled", [False, True])
def test_batch_measurements_equal_plain_observables(pooled):
    from chllmodel_b200.batched import Batch
    from chllmodel_b200.lattice import Lattice, coupling
    from chllmodel_b200.observables import nematic_S

    specs = _specs()
    with Batch(specs) as b:
        b.set_tuning(256, 0, pooled=pooled)
        b.init_random()
        b.run(10, measure_every=10)
        mom = b.moments()
        for r, sp in enumerate(specs):
            lat = Lattice(sp["ni"], sp["nj"], sp["nk"], boundary=sp["boundary"])
            lat.upload_f4(b.download_f4(r))
            row = lat.observe(coupling(sp["kT"], sp["K"], sp["g"], sp["eps"]))
            n = sp["ni"] * sp["nj"] * sp["nk"]
            assert mom[r, 0] == 1
            assert mom[r, 8] == pytest.approx(row[5] / n, rel=1e-12, abs=1e-12)
            assert mom[r, 9] == pytest.approx(row[6] / n, rel=1e-12, abs=1e-12)
            assert mom[r, 10] == pytest.approx(nematic_S(row[7:13], n), rel=1e-10, abs=1e-12)
            assert mom[r, 15] == 0
            lat.close()


def test_batch_k0_field_limit():
    """K = 0: <s> = tanh(g/kT) for every replica of a field grid."""
    from chllmodel_b200.batched import Batch, replica

    kT = 1.0
    gs = [0.0, 0.1, 0.25, 0.5, 1.0]
    specs = [replica(16, kT=kT, K=0.0, g=g, seed=11 + i, replica=i) for i, g in enumerate(gs)]
    with Batch(specs) as b:
        b.init_random()
        # odd interval: at g = 0 every flip has dE = 0 and is always accepted
        # (chll_mod.f90:235), so eta alternates sign each sweep
        b.run(1200, measure_every=3, measure_from=200)
        summ = b.summary()
    for sp, s in zip(specs, summ):
        m = s["n_meas"]
        # a single spin's variance bounds the per-site variance of eta
        se = math.sqrt((1 - math.tanh(sp["g"] / kT) ** 2) / (16 ** 3 * m))
        # successive measurements are correlated: allow a generous factor
        assert abs(s["eta"] - math.tanh(sp["g"] / kT)) < 6 * se * 3 + 2e-3


def test_batch_autotune_restores_state():
    from chllmodel_b200.batched import Batch

    specs = _specs()
    with Batch(specs) as b:
        b.init_random()
        b.run(3, measure_every=0)
        before = [b.download_f4(r) for r in range(len(specs))]
        mom_before = b.moments()
        res = b.autotune(trial_sweeps=2)
        assert res["threads"] in (128, 256, 512) and res["ctas_per_sm"] >= 1
        after = [b.download_f4(r) for r in range(len(specs))]
        for x, y in zip(before, after):
            assert np.array_equal(x, y)
        assert np.array_equal(b.moments(), mom_before)
        info = b.info()
        assert info["threads"] == res["threads"] and info["grid"] >= len(specs)


def test_batch_rejects_bad_specs():
    from chllmodel_b200 import _lib
    from chllmodel_b200.batched import Batch, replica

    with pytest.raises(_lib.ChllError, match="odd"):
        Batch([replica(7, kT=1.0, K=1.0, boundary="periodic")])
    with pytest.raises(_lib.ChllError, match="kT"):
        Batch([replica(8, kT=-1.0, K=1.0)])


def test_batch_barrier_wait_gives_up():
    """A group-barrier wait limited to one poll runs out on a replica of many
    CTAs: its status word is set, its CTAs leave the launch, the one-CTA
    replica (which never waits) finishes every sweep, chll_batch_moments
    reports CHLL_EDEVICE, and the context stays usable."""
    import ctypes as ct

    from chllmodel_b200 import _lib
    from chllmodel_b200.batched import Batch, replica

    L = _lib.load()
    nsw = 40
    specs = [replica(64, kT=0.5, K=1.0, seed=3, replica=0),
             replica(8, kT=0.5, K=1.0, seed=4, replica=1)]
    with Batch(specs) as b:
        b.set_tuning(128, 0, paired=False)  # each replica its own group
        assert b.info()["grid"] > 2  # the 64^3 replica spans many CTAs
        b.init_random()
        b.set_wait_limit(1)
        b.run(nsw, measure_every=10)
        m = np.zeros((2, 16), np.float64)
        rc = L.chll_batch_moments(b._h, m.ctypes.data_as(ct.c_void_p))
        assert rc == _lib.CHLL_EDEVICE
        assert "timed out" in _lib.last_error()
        assert m[0, 15] != 0
        assert m[1, 15] == 0 and int(m[1, 12]) == nsw + 1
    with pytest.raises(_lib.ChllError):
        Batch(specs).set_wait_limit(0)
    # a new batch with the default limit runs cleanly on the same context
    with Batch(specs) as b:
        b.init_random()
        b.run(4, measure_every=2)
        m = b.moments()
        assert np.all(m[:, 15] == 0) and np.all(m[:, 12] == 5)
