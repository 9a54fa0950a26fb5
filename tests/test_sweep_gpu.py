"""GPU parity of the checkerboard sweep against the oracle.

Lockstep protocol: before each half-sweep the oracle reads the GPU's FP32
state (exactly, as FP64) and runs the same pass on the same Philox stream
with the reference's arithmetic.  Then
  * accept/reject decisions and chiralities agree bit for bit except at
    logged near-threshold ties, |dE_ref - (-kT ln u)| <= TIE_DE;
  * accepted directors agree within DIR_RTOL (relative, per vector);
  * everything not of the pass's colour is untouched.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TIE_DE = 2e-5      # |enew-eold| error bound of two FP32 energy evaluations
DIR_RTOL = 1e-5    # director tolerance of the FP32 trial vs the FP64 trial
ENERGY_RTOL = 1e-6


def _decisions_gpu(before, after, p):
    if p < 2:
        return np.any(np.stack([a != b for a, b in zip(before[:3], after[:3])]), axis=0)
    return before[3] != after[3]


def lockstep(oracle, shape, periodic, kT, K, g, eps=1.0, sweeps=3, seed=5, d0=0.1,
             init_seed=3):
    from chllmodel_b200.lattice import Lattice, coupling

    cfg = oracle.make_cfg(*shape, periodic=periodic, kT=kT, K=K, g=g, eps=eps, seed=seed)
    icfg = oracle.make_cfg(*shape, seed=init_seed)
    nx, ny, nz, s = oracle.init_random(icfg)
    lat = Lattice(*shape, boundary="periodic" if periodic else "open")
    lat.upload_f64(nx, ny, nz, s)
    lat.set_control(d0, step=1)
    cp = coupling(kT, K, g, eps)
    ties = 0
    decided = 0
    ni, nj, nk = shape
    parity = ((np.arange(ni, dtype=np.int32)[:, None, None] +
               np.arange(nj, dtype=np.int32)[None, :, None] +
               np.arange(nk, dtype=np.int32)[None, None, :]) & 1).astype(np.int8)
    for _ in range(sweeps):
        for p in range(4):
            ctl = lat.control()
            state = lat.download_f64()
            before = [a.copy(order="F") for a in state]
            lat.half_sweep(cp, p, seed=seed)
            after = lat.download_f64()
            onx, ony, onz, os_ = [a.copy(order="F") for a in before]
            d32 = float(np.float32(ctl["d"]))
            n, acc, de, u = oracle.run_pass(cfg, p, ctl["step"], d32, onx, ony, onz, os_,
                                            detail=True)
            mine = parity == (p & 1)
            # untouched colour
            for a, b in zip(after, before):
                assert np.array_equal(a[~mine], b[~mine])
            gdec = _decisions_gpu(before, after, p)
            odec = acc == 1
            mism = mine & (gdec != odec)
            if mism.any():
                thr = np.where(u > 0, -kT * np.log(np.where(u > 0, u, 1.0)), np.inf)
                gap = np.abs(de - thr)
                assert np.all(gap[mism] <= TIE_DE), (
                    f"pass {p}: {int(mism.sum())} decision mismatches, gaps {gap[mism][:5]}")
                ties += int(mism.sum())
            decided += int(mine.sum())
            both = mine & gdec & odec
            if p < 2:
                gv = np.stack([after[0], after[1], after[2]], -1)[both]
                ov = np.stack([onx, ony, onz], -1)[both]
                err = np.linalg.norm(gv - ov, axis=-1) / np.linalg.norm(ov, axis=-1)
                assert err.max(initial=0.0) <= DIR_RTOL
            else:
                assert np.array_equal(after[3][both], os_[both])
    lat.close()
    return ties, decided


CASES = [
    # shape, periodic, kT, K, g, eps
    ((8, 8, 8), False, 0.5, 0.5, 0.0, 1.0),
    ((8, 8, 8), True, 0.5, 1.0, 0.25, 1.0),
    ((7, 6, 5), False, 0.8, 0.7, 0.1, 1.0),     # odd ni: padded storage
    ((6, 4, 8), True, 0.3, 1.0, 0.5, 1.0),      # ni = 2 mod 4, periodic
    ((12, 10, 6), False, 1.5, 1.0, 3.0, 0.7),   # large field, eps != 1
    ((1, 5, 3), False, 0.5, 0.5, 0.0, 1.0),     # single column
    ((16, 16, 16), True, 0.1, 1.0, 0.0, 1.0),   # cold: small acceptance
]


@pytest.mark.parametrize("shape,periodic,kT,K,g,eps", CASES)
def test_lockstep_half_sweeps(oracle, shape, periodic, kT, K, g, eps):
    ties, decided = lockstep(oracle, shape, periodic, kT, K, g, eps)
    assert ties <= max(2, decided // 2000)


@pytest.mark.parametrize("periodic", [False, True])
def test_lockstep_reference_size_run(oracle, periodic):
    """The 32^3 reference-size configuration itself (K = 0.5, h = 0,
    kT = 0.5, d0 = 0.1, seed 1 for the initial state and the sweeps), open
    as the reference's sweep and periodic, four sweeps in lockstep; then the
    library's fused sweep from the same start reaches the four half-sweeps'
    final GPU state and control block bit for bit."""
    shape, nsw = (32, 32, 32), 4
    ties, decided = lockstep(oracle, shape, periodic, 0.5, 0.5, 0.0, sweeps=nsw, seed=1,
                             d0=0.1, init_seed=1)
    assert decided == 32 ** 3 * 2 * nsw
    assert ties <= max(2, decided // 2000)
    assert _fused_equals_half_sweeps(oracle, shape, periodic, 0.5, 0.5, 0.0, nsw, 1)


def _fused_equals_half_sweeps(oracle, shape, periodic, kT, K, g, nsw, seed, d0=0.1):
    """From the oracle's initial state, the library's fused sweep (the column
    walk where ni is a multiple of 4) and the four half-sweep kernels reach
    the same state and control block bit for bit after nsw sweeps."""
    from chllmodel_b200.lattice import Lattice, coupling

    bnd = "periodic" if periodic else "open"
    nx, ny, nz, s = oracle.init_random(oracle.make_cfg(*shape, seed=seed))
    four, fused = Lattice(*shape, boundary=bnd), Lattice(*shape, boundary=bnd)
    fused.set_kernel("fused")
    cp = coupling(kT, K, g)
    for lat in (four, fused):
        lat.upload_f64(nx, ny, nz, s)
        lat.set_control(d0, step=1)
    for _ in range(nsw):
        for p in range(4):
            four.half_sweep(cp, p, seed=seed)
    fused.sweep(cp, nsw, seed=seed)
    same = np.array_equal(four.download_f4(), fused.download_f4())
    ctl = four.control() == fused.control()
    four.close()
    fused.close()
    return same and ctl


# The other workloads' own lattices and couplings (eps = 1): the 128^3
# anneal (K = 1, h = 0.25, seed 7) at its first and last stage temperatures,
# periodic, and its first stage with the reference's own open boundaries (the
# default of ChLLSim); the 64^3 differentiation workload's equilibration
# (kT 0.3, K = 1, h = 0.5, seed 3) and a 48^3 replica at two corners of the
# batched phase grid (K = 1; kT 0.1, h 3.0 and kT 2.0, h 0.0), periodic.
WORKLOAD_CASES = [
    ((128, 128, 128), True, 1.5, 1.0, 0.25, 7, 2),
    ((128, 128, 128), True, 0.1, 1.0, 0.25, 7, 2),
    ((128, 128, 128), False, 1.5, 1.0, 0.25, 7, 2),
    ((64, 64, 64), True, 0.3, 1.0, 0.5, 3, 3),
    ((48, 48, 48), True, 0.1, 1.0, 3.0, 2, 3),
    ((48, 48, 48), True, 2.0, 1.0, 0.0, 2, 3),
]


@pytest.mark.parametrize("shape,periodic,kT,K,g,seed,nsw", WORKLOAD_CASES)
def test_lockstep_workload_lattices(oracle, shape, periodic, kT, K, g, seed, nsw):
    """Lockstep against the oracle on the workloads' own lattice sizes and
    couplings, then the fused sweep from the same start equal to the four
    half-sweeps bit for bit."""
    ties, decided = lockstep(oracle, shape, periodic, kT, K, g, sweeps=nsw, seed=seed, d0=0.1,
                             init_seed=seed)
    assert decided == int(np.prod(shape)) * 2 * nsw
    assert ties <= max(2, decided // 2000)
    assert _fused_equals_half_sweeps(oracle, shape, periodic, kT, K, g, nsw, seed)


def test_lockstep_benchmark_lattice(oracle):
    """The 480^3 benchmark lattice itself (periodic, K = 1, h = 0, kT = 0.3,
    seed 11): one sweep in lockstep with the oracle (110.6 M sites), then one
    fused sweep -- the benchmark's column-walk kernels -- equal to the four
    half-sweep kernels bit for bit."""
    shape = (480, 480, 480)
    ties, decided = lockstep(oracle, shape, True, 0.3, 1.0, 0.0, sweeps=1, seed=11, d0=0.1,
                             init_seed=11)
    assert decided == 480 ** 3 * 2
    assert ties <= max(2, decided // 2000)
    assert _fused_equals_half_sweeps(oracle, shape, True, 0.3, 1.0, 0.0, 1, 11)


@pytest.mark.parametrize("shape,periodic", [((32, 32, 32), True), ((32, 32, 32), False),
                                            ((48, 48, 48), True), ((30, 18, 10), False)])
def test_resident_form_follows_the_chain(oracle, shape, periodic):
    """The resident form (a chunk of sweeps in one cluster launch) on the
    small workload sizes: the 32^3 configuration's couplings, chunks of 100
    and 37 sweeps with a measurement row after each, equal to the fused
    passes' state, control block and rows bit for bit."""
    from chllmodel_b200.lattice import Lattice, coupling

    nx, ny, nz, s = oracle.init_random(oracle.make_cfg(*shape, seed=1))
    cp = coupling(0.5, 0.5, 0.0)
    out = []
    for kind in ("fused", "resident"):
        lat = Lattice(*shape, boundary="periodic" if periodic else "open")
        lat.set_kernel(kind)
        lat.upload_f64(nx, ny, nz, s)
        lat.set_control(0.1, step=1)
        lat.reserve_rows(3)
        for r, n in enumerate((100, 37, 100)):
            lat.sweep(cp, n, seed=1)
            lat.measure(cp, r)
        out.append((lat.download_f4(), lat.control(), lat.read_rows(0, 3)))
        lat.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])


def test_zero_temperature_rule(oracle):
    ties, decided = lockstep(oracle, (8, 8, 6), False, 0.0, 1.0, 0.5, sweeps=2)
    assert ties <= 2


def test_device_init_matches_oracle(oracle):
    from chllmodel_b200.lattice import Lattice

    shape = (10, 7, 5)
    lat = Lattice(*shape)
    lat.init_random(seed=42, replica=3)
    nx, ny, nz, s = lat.download_f64()
    cfg = oracle.make_cfg(*shape, seed=42, replica=3)
    ox, oy, oz, os_ = oracle.init_random(cfg)
    assert np.array_equal(s, os_)
    assert np.max(np.abs(nx - ox)) < 1e-6 and np.max(np.abs(ny - oy)) < 1e-6
    assert np.max(np.abs(nz - oz)) < 1e-7
    lat.close()


@pytest.mark.parametrize("shape", [(8, 8, 8), (7, 5, 3), (13, 4, 6), (2, 2, 2)])
def test_layout_roundtrip(shape):
    from chllmodel_b200.lattice import Lattice, to_f4

    rng = np.random.default_rng(0)
    nx, ny, nz = (np.asfortranarray(rng.normal(size=shape)) for _ in range(3))
    s = np.asfortranarray(np.where(rng.random(shape) < 0.5, -1, 1).astype(np.int32))
    lat = Lattice(*shape)
    lat.upload_f64(nx, ny, nz, s)
    bx, by, bz, bs = lat.download_f64()
    assert np.array_equal(bx, nx.astype(np.float32).astype(np.float64))
    assert np.array_equal(bz, nz.astype(np.float32).astype(np.float64))
    assert np.array_equal(bs, s)
    f4 = lat.download_f4()
    assert np.array_equal(f4, to_f4(nx, ny, nz, s))
    lat.upload_f4(f4[::-1].copy())
    assert np.array_equal(lat.download_f4(), f4[::-1])
    lat.close()


@pytest.mark.parametrize("periodic", [False, True])
def test_energy_observables_match_fp64_oracle(oracle, periodic):
    from chllmodel_b200.lattice import Lattice, coupling

    shape = (16, 12, 10)
    lat = Lattice(*shape, boundary="periodic" if periodic else "open")
    lat.init_random(seed=7)
    cp = coupling(0.5, 1.0, 0.25, 1.0)
    lat.set_control(0.1, step=1)
    lat.sweep(cp, 20, seed=11)
    row = lat.observe(cp)
    nx, ny, nz, s = lat.download_f64()
    cfg = oracle.make_cfg(*shape, periodic=periodic, K=1.0, g=0.25)
    mo = oracle.moments(cfg, nx, ny, nz, s)
    assert row[5] == pytest.approx(mo[0], rel=ENERGY_RTOL)
    assert row[13] == pytest.approx(mo[1], rel=ENERGY_RTOL)
    assert row[6] == mo[2]
    np.testing.assert_allclose(row[7:13], mo[3:9], rtol=1e-9, atol=1e-9)
    v32, _ = oracle.etot(cfg, nx, ny, nz, s, mode=0)
    assert row[0] == pytest.approx(v32, rel=1e-6)
    ctl = lat.control()
    assert row[2] == ctl["paccept"] and row[4] == ctl["d"]
    lat.close()


def test_step_epilogue_on_device(oracle):
    """paccept/faccept/d adaptation/step counter run on the device."""
    from chllmodel_b200.lattice import Lattice, coupling

    shape = (16, 16, 16)
    lat = Lattice(*shape)
    lat.init_random(seed=1)
    lat.set_control(0.1, step=1, adapt_until=10000)
    cp = coupling(0.5, 0.5, 0.0)
    d = 0.1
    for sweep in range(1, 6):
        lat.sweep(cp, 1, seed=2)
        ctl = lat.control()
        assert ctl["step"] == sweep + 1
        pa = ctl["paccept"]
        assert pa == float(np.float32(pa))
        f = float(np.float32(0.995))
        d = d * f if pa < 0.4 else (d / f if pa > 0.6 else d)
        assert ctl["d"] == d
    # no adaptation at or beyond adapt_until
    lat.set_control(0.2, step=50, adapt_until=50)
    lat.sweep(cp, 3, seed=2)
    assert lat.control()["d"] == 0.2
    lat.close()


def test_graph_replay_equals_single_passes(oracle):
    """A captured multi-sweep graph gives the same state as pass-by-pass."""
    from chllmodel_b200.lattice import Lattice, coupling

    shape = (12, 8, 8)
    cp = coupling(0.6, 1.0, 0.1)
    a, b = Lattice(*shape), Lattice(*shape)
    for lat in (a, b):
        lat.init_random(seed=5)
        lat.set_control(0.1, step=1)
    a.sweep(cp, 7, seed=9)
    for _ in range(7):
        for p in range(4):
            b.half_sweep(cp, p, seed=9)
    assert np.array_equal(a.download_f4(), b.download_f4())
    assert a.control() == b.control()
    a.close()
    b.close()


@pytest.mark.parametrize("shape,periodic", [((16, 16, 16), True), ((24, 10, 6), False),
                                            ((7, 9, 5), False), ((6, 4, 8), True),
                                            ((120, 6, 4), True), ((64, 64, 4), False)])
def test_sweep_forms_follow_one_chain(shape, periodic):
    """The fused two-pass sweep, the four half-sweeps of the direct kernel,
    the staged kernel, the resident cluster launch, four single
    chll_lattice_pass calls per sweep and the fused passes issued one by one
    all follow one chain bit for bit (same units, counters and arithmetic),
    with the same control block (d, step, paccept, faccept)."""
    from chllmodel_b200.lattice import FUSED_A, FUSED_A0, FUSED_B, FUSED_F, Lattice, coupling

    cp = coupling(0.6, 1.0, 0.2, 1.1)
    out = []
    for kind in ("fused", "direct", "staged", "resident", "passes", "fused_passes"):
        lat = Lattice(*shape, boundary="periodic" if periodic else "open")
        if kind not in ("passes", "fused_passes"):
            lat.set_kernel(kind)
        lat.init_random(seed=21)
        lat.set_control(0.15, step=1)
        if kind == "passes":
            for _ in range(9):
                for p in range(4):
                    lat.half_sweep(cp, p, seed=4)
        elif kind == "fused_passes":
            seq = [FUSED_A0, FUSED_B] + [FUSED_A, FUSED_B] * 8 + [FUSED_F]
            for p in seq:
                lat.half_sweep(cp, p, seed=4)
        else:
            lat.sweep(cp, 4, seed=4)
            lat.sweep(cp, 5, seed=4)  # a second call: flips closed in between
        out.append((lat.download_f4(), lat.control()))
        lat.close()
    for state, ctl in out[1:]:
        assert np.array_equal(out[0][0], state)
        assert out[0][1] == ctl
