"""GPU tests of the workflow drivers: annealing keeps the lattice on the
device and orders it as kT falls; the batched phase diagram returns every
point; ChLLSim.run through the reference entry point prints the reference
table and fills msteps/m with the reference semantics."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_anneal_orders_the_lattice():
    from chllmodel_b200.lattice import Lattice
    from chllmodel_b200.workflows import anneal, linear_schedule

    # K = 0: the Lebwohl-Lasher nematic orders (S -> ~0.96 at kT = 0.1 on the
    # oracle).  K = 1 with a field: the chirality deracemises (eta -> 1) while
    # the cholesteric twist keeps the global S small.
    for K in (0.0, 1.0):
        lat = Lattice(16, 16, 16, boundary="periodic")
        lat.init_random(7)
        stages = anneal(lat, linear_schedule(1.5, 0.1, 5), 300, K=K, g=0.25, seed=7, d0=0.1)
        assert [round(s["kT"], 3) for s in stages] == [1.5, 1.15, 0.8, 0.45, 0.1]
        assert stages[-1]["step"] == 1 + 5 * 300
        es = [s["energy"] for s in stages]
        assert all(b < a for a, b in zip(es, es[1:]))
        if K == 0.0:
            assert stages[0]["S"] < 0.1 and stages[-1]["S"] > 0.8
        else:
            assert stages[-1]["abs_eta"] > 0.9
        lat.close()


def test_phase_diagram_batch():
    from chllmodel_b200.workflows import phase_diagram

    res = phase_diagram([0.3, 1.5], [0.0, 2.0], [8, 12], nsweeps=200, measure_every=5,
                        measure_from=100, autotune=False)
    assert len(res) == 4
    for r in res:
        assert r["n_meas"] == 21 and np.isfinite(r["energy"])  # sweeps 100, 105, ..., 200
    hot_field = [r for r in res if r["kT"] == 1.5 and r["g"] == 2.0][0]
    assert hot_field["eta"] > 0.5


def test_chllsim_reference_run(capfd, oracle):
    from chllmodel_b200 import chll

    chll.set_seed(5)
    sim = chll.ChLLSim(12, 12, 12, 0.5, 0.1, 0.5, 0.1, 0.0)
    sim.init_random_directors(np.random.RandomState(3))
    sim.init_rand_s()
    sim.run(300, 100)
    out = capfd.readouterr().out.splitlines()
    hdr = [i for i, l in enumerate(out) if l.startswith("Steps ")]
    assert hdr and out[hdr[0]] == "Steps       Energy      E. excess      Paccept      Faccept      D"
    rows = out[hdr[0] + 1:hdr[0] + 4]
    assert [int(r[:8]) for r in rows] == [100, 200, 300]
    assert all(len(r) == 8 + 5 * 13 for r in rows)
    assert list(sim.msteps) == [100, 200, 300]
    assert sim.m.flags["F_CONTIGUOUS"] and sim.m.shape == (3, 5)
    # last row describes the final state, with the reference's etot semantics
    cfg = oracle.make_cfg(12, 12, 12, K=0.5, g=0.1)
    v32, _ = oracle.etot(cfg, sim.nx, sim.ny, sim.nz, sim.s, mode=0)
    assert sim.m[2, 0] == pytest.approx(v32, rel=1e-6)
    assert sim.m[2, 1] == np.float32(np.float32(sim.s.sum()) / np.float32(12 ** 3))
    assert sim.m[2, 4] == sim.d
    assert float(rows[-1].split()[5]) == pytest.approx(sim.d, abs=1e-6)
    # the Fortran layout of directors is kept and they stay unit vectors
    assert sim.nx.flags["F_CONTIGUOUS"]
    assert np.allclose(sim.nx ** 2 + sim.ny ** 2 + sim.nz ** 2, 1.0, atol=1e-5)


def test_chllsim_resume_is_exact(tmp_path):
    """Seed, step and d in the NPZ make a split run equal an unsplit one."""
    from chllmodel_b200 import chll

    def make(name):
        s = chll.ChLLSim(8, 8, 8, 0.6, 0.1, 1.0, 0.2, 0.0, name=name, data_folder=str(tmp_path),
                         seed=9, boundary="periodic", verbose=False)
        s.init_random_directors(np.random.RandomState(1))
        s.s[:] = np.where(np.random.RandomState(2).rand(8, 8, 8) < 0.5, -1, 1)
        return s

    a = make("a")
    a.run(200, 50)
    b = make("b")
    b.run(120, 40, save=True)
    c = chll.ChLLSim(8, 8, 8, 0.6, 0.1, 1.0, 0.2, 0.0, name="c", data_folder=str(tmp_path),
                     seed=9, boundary="periodic", verbose=False)
    s = c.load_config(str(tmp_path / "b" / "b_data.npz"))
    c.s[:] = s
    c.run(80, 40, nstart=c.step + 1)
    assert np.array_equal(a.nx, c.nx) and np.array_equal(a.s, c.s)
    assert a.d == c.d


def test_uniform_start_of_a_batch():
    """init_uniform gives every site the director (normalised) and +-1 spins;
    an aligned start at low temperature without chiral coupling stays
    nematically ordered, as the reference drivers' init_aligned2 runs."""
    from chllmodel_b200.batched import Batch, replica
    from chllmodel_b200.workflows import phase_diagram

    specs = [replica(8, kT=0.5, K=1.0, seed=3, replica=0), replica(6, 4, 10, kT=0.5, K=1.0,
                                                                    seed=4, replica=1)]
    with Batch(specs) as b:
        b.init_uniform((2.0, 0.0, 2.0))
        for r in range(len(specs)):
            st = b.download_f4(r)
            want = np.array([np.sqrt(0.5), 0.0, np.sqrt(0.5)], np.float32)
            assert np.array_equal(st[:, :3], np.broadcast_to(want, st[:, :3].shape))
            assert set(np.unique(st[:, 3])) == {-1.0, 1.0}
    res = phase_diagram([0.1], [0.0], [12], K=0.0, nsweeps=60, measure_every=10,
                        autotune=False, init="aligned2")
    assert res[0]["S"] > 0.9
