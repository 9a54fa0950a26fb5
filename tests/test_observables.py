"""CPU tests of the derived observables (S, C_v, chi_c) and the phase-grid
builder."""
import math

import numpy as np
import pytest

from chllmodel_b200 import observables as ob
from chllmodel_b200.batched import phase_grid, replica


def sums6(n):
    n = np.asarray(n, dtype=np.float64)
    x, y, z = n[:, 0], n[:, 1], n[:, 2]
    return [np.sum(x * x), np.sum(y * y), np.sum(z * z), np.sum(x * y), np.sum(x * z),
            np.sum(y * z)]


def test_nematic_S_limits():
    aligned = np.tile([0.0, 0.6, 0.8], (1000, 1))
    assert ob.nematic_S(sums6(aligned), 1000) == pytest.approx(1.0, abs=1e-12)
    # directors uniform in a plane (a full cholesteric turn): S = 1/4
    phi = np.linspace(0, 2 * np.pi, 4000, endpoint=False)
    planar = np.stack([np.cos(phi), np.sin(phi), 0 * phi], 1)
    assert ob.nematic_S(sums6(planar), 4000) == pytest.approx(0.25, abs=1e-12)
    rng = np.random.default_rng(0)
    v = rng.normal(size=(200000, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    assert ob.nematic_S(sums6(v), len(v)) < 0.01


def test_fluctuation_formulas():
    rng = np.random.default_rng(1)
    e = rng.normal(1.0, 0.01, 5000)
    kT, n = 0.5, 4096
    assert ob.specific_heat(e, kT, n) == pytest.approx(n * e.var() / kT ** 2)
    assert ob.specific_heat_reference(e, kT) == pytest.approx(e.var() / kT)
    eta = rng.normal(0.2, 0.05, 5000)
    assert ob.chiral_susceptibility(eta, kT, n) == pytest.approx(n * eta.var() / kT)
    assert ob.chiral_susceptibility(eta, kT, n, reference_form=False) == pytest.approx(eta.var())


def test_summarize_batch_moments():
    specs = [replica(8, kT=0.5, K=1.0, g=0.1)]
    e = np.array([1.0, 1.2, 0.8, 1.0])
    eta = np.array([0.1, -0.1, 0.3, 0.1])
    S = np.array([0.2, 0.3, 0.25, 0.25])
    row = np.zeros((1, 16))
    row[0, :8] = [4, e.sum(), (e * e).sum(), eta.sum(), (eta * eta).sum(), np.abs(eta).sum(),
                  S.sum(), (S * S).sum()]
    out = ob.summarize_batch(row, specs)[0]
    n = 512
    assert out["energy"] == pytest.approx(1.0)
    assert out["C_v"] == pytest.approx(n * e.var() / 0.25)
    assert out["chi_c"] == pytest.approx(n * eta.var() / 0.5)
    assert out["S"] == pytest.approx(0.25) and out["abs_eta"] == pytest.approx(0.15)


def test_phase_grid_is_the_batched_config():
    kTs = np.linspace(0.1, 2.0, 8)
    gs = np.linspace(0.0, 3.0, 8)
    specs = phase_grid(kTs, gs, [32, 48, 64], K=1.0, seed=1)
    assert len(specs) == 64
    assert {s["ni"] for s in specs} <= {32, 48, 64} and len({s["ni"] for s in specs}) == 3
    assert all(s["ni"] == s["nj"] == s["nk"] for s in specs)
    assert [s["seed"] for s in specs] == [1 + i for i in range(64)]
    assert sorted({round(s["kT"], 6) for s in specs}) == [round(x, 6) for x in kTs]
    assert sorted({round(s["g"], 6) for s in specs}) == [round(x, 6) for x in gs]
    assert phase_grid(kTs, gs, [32, 48, 64], seed=1) == specs
    assert all(math.isclose(s["K"], 1.0) and s["boundary"] == "periodic" for s in specs)


def test_fluctuations_match_the_reference_measure_chi(golden_dir, tmp_path):
    """chll.ChLLSim writes the reference's macro CSV (Step,TotalEnergy,
    Eexcess,Paccept,Faccept,D); the reference's measure_chi
    (notebooks/.ipynb_checkpoints/Xch-checkpoint.ipynb, cell 2) read seeded
    files of that format (tests/golden/chi_golden.npz, generated by running it).
    The fluctuation formulas of chllmodel_b200.observables in their reference
    forms give its numbers, and a file written by save_macros reads back to
    the rows it holds."""
    import os

    import numpy as np

    from chllmodel_b200 import chll
    from chllmodel_b200 import observables as ob

    d = np.load(os.path.join(golden_dir, "chi_golden.npz"))
    pts = [tuple(p) for p in d["points"]]
    for K in sorted({p[0] for p in pts}):
        got_chi, got_ex, got_cv = [], [], []
        for q, (k, kbt) in enumerate(pts):
            if k != K:
                continue
            rows = d[f"p{q}_rows"]
            got_chi.append(ob.chiral_susceptibility(rows[:, 2], kbt, 1, reference_form=False))
            got_ex.append(float(np.mean(rows[:, 2])))
            got_cv.append(ob.specific_heat_reference(rows[:, 1], kbt))
        np.testing.assert_allclose(got_chi, d[f"K{K}_chi"], rtol=1e-12)
        np.testing.assert_allclose(got_ex, d[f"K{K}_excess"], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(got_cv, d[f"K{K}_cv"], rtol=1e-12)
    # the CSV that ChLLSim writes is the file measure_chi reads
    sim = chll.ChLLSim(4, 4, 4, 0.5, 0.1, 1.0, 0.0, 0.0, name="csvcheck", overwrite=True,
                       verbose=False, data_folder=str(tmp_path))
    rows = d["p0_rows"]
    sim.msteps = rows[:, 0].astype(np.int32)
    sim.m = np.asfortranarray(rows[:, 1:6])
    sim.save_macros()
    back = np.loadtxt(os.path.join(sim.simpath, "csvcheck.csv"), skiprows=1, delimiter=",")
    np.testing.assert_array_equal(back, rows)
