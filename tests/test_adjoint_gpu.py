"""GPU parity of the energy adjoint kernel: dE/dn_i for every director
(raw and tangent-projected) and dE/d(eps, K, h), against the FP64 oracle
gradient on the same FP32 state and against central finite differences of
the FP64 total energy."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRAD_RTOL = 2e-5   # FP32 per-site sum of six bond terms vs FP64
GRAD_ATOL = 2e-5


@pytest.mark.parametrize("shape,periodic", [((12, 10, 8), True), ((9, 7, 5), False),
                                            ((6, 6, 4), True)])
@pytest.mark.parametrize("project", [False, True])
def test_gradient_matches_fp64_oracle(oracle, shape, periodic, project):
    from chllmodel_b200.lattice import Lattice, coupling

    lat = Lattice(*shape, boundary="periodic" if periodic else "open")
    lat.init_random(seed=3)
    cp = coupling(0.3, 1.0, 0.5, 1.2)
    lat.set_control(0.1, step=1)
    lat.sweep(cp, 5, seed=3)
    g, out4 = lat.energy_grad(cp, project=project)
    nx, ny, nz, s = lat.download_f64()
    cfg = oracle.make_cfg(*shape, periodic=periodic, K=1.0, g=0.5, eps=1.2)
    og, oout = oracle.energy_grad(cfg, nx, ny, nz, s, project=project)
    og = np.stack([og[..., c].ravel(order="F") for c in range(3)], 1)
    g3 = g[:, :3].astype(np.float64)
    np.testing.assert_allclose(g3, og, rtol=GRAD_RTOL, atol=GRAD_ATOL)
    assert np.all(g[:, 3] == 0)
    np.testing.assert_allclose(out4, oout, rtol=1e-9, atol=1e-9)
    if project:
        n = np.stack([nx.ravel(order="F"), ny.ravel(order="F"), nz.ravel(order="F")], 1)
        assert np.max(np.abs(np.sum(g3 * n, 1))) < 1e-5
    lat.close()


def test_gradient_central_differences(oracle):
    """Central differences (step 1e-3) of the FP64 total energy on random
    sites of a 64^3 lattice equilibrated at kT = 0.3."""
    from chllmodel_b200.lattice import Lattice, coupling

    shape = (64, 64, 64)
    lat = Lattice(*shape, boundary="periodic")
    lat.init_random(seed=3)
    cp = coupling(0.3, 1.0, 0.5, 1.0)
    lat.set_control(0.1, step=1)
    lat.sweep(cp, 50, seed=3)
    g, out4 = lat.energy_grad(cp)
    nx, ny, nz, s = lat.download_f64()
    cfg = oracle.make_cfg(*shape, periodic=True, K=1.0, g=0.5, eps=1.0)
    h = 1e-3
    rng = np.random.default_rng(0)
    sites = rng.integers(0, 64, size=(1000, 3))
    for (i, j, k) in sites:
        e_idx = i + 64 * (j + 64 * k)
        for comp, arr in enumerate((nx, ny, nz)):
            old = arr[i, j, k]
            # the local energy holds every term that depends on this director
            arr[i, j, k] = old + h
            ep = oracle.site_energy(cfg, nx, ny, nz, s, int(i), int(j), int(k))
            arr[i, j, k] = old - h
            em = oracle.site_energy(cfg, nx, ny, nz, s, int(i), int(j), int(k))
            arr[i, j, k] = old
            fd = (ep - em) / (2 * h)
            # site_energy accumulates in FP32: ~1e-6 absolute per evaluation
            assert g[e_idx, comp] == pytest.approx(fd, abs=5e-3)
    lat.close()


def test_gradient_quench_lowers_energy():
    """Zero-temperature gradient descent along the tangent-projected gradient
    (director renormalised) lowers the energy monotonically."""
    from chllmodel_b200.lattice import Lattice, coupling

    shape = (16, 16, 16)
    lat = Lattice(*shape, boundary="periodic")
    lat.init_random(seed=9)
    cp = coupling(0.0, 1.0, 0.5, 1.0)
    energies = []
    for _ in range(30):
        g, out4 = lat.energy_grad(cp, project=True)
        energies.append(out4[0])
        f4 = lat.download_f4()
        f4[:, :3] -= 0.05 * g[:, :3]
        f4[:, :3] /= np.linalg.norm(f4[:, :3], axis=1, keepdims=True)
        lat.upload_f4(f4)
    assert all(b <= a + 1e-6 for a, b in zip(energies, energies[1:]))
    assert energies[-1] < energies[0] - 0.1 * abs(energies[0])
    lat.close()


@pytest.mark.parametrize("shape,periodic", [((12, 10, 8), True), ((9, 7, 5), False),
                                            ((6, 6, 4), True)])
def test_quench_step_matches_fp64_gradient(oracle, shape, periodic):
    """One quench step on the device (colour 0, then colour 1 with colour 0
    already moved) against n <- normalise(n - eta * projected FP64 gradient)
    of the oracle, colour by colour; chiralities unchanged."""
    from chllmodel_b200.lattice import Lattice, coupling

    eta = 0.05
    lat = Lattice(*shape, boundary="periodic" if periodic else "open")
    lat.init_random(seed=5)
    cp = coupling(0.3, 1.0, 0.5, 1.2)
    lat.set_control(0.1, step=1)
    lat.sweep(cp, 3, seed=5)
    nx, ny, nz, s = lat.download_f64()
    cfg = oracle.make_cfg(*shape, periodic=periodic, K=1.0, g=0.5, eps=1.2)
    i, j, k = np.indices(shape)
    colour = (i + j + k) & 1
    cur = [a.copy(order="F") for a in (nx, ny, nz)]
    for c in (0, 1):
        og, _ = oracle.energy_grad(cfg, cur[0], cur[1], cur[2], s, project=True)
        new = [a - eta * og[..., m] for m, a in enumerate(cur)]
        norm = np.sqrt(new[0] ** 2 + new[1] ** 2 + new[2] ** 2)
        mask = colour == c
        for m in range(3):
            cur[m] = np.asfortranarray(np.where(mask, new[m] / norm, cur[m]))
    lat.quench(cp, eta, 1)
    gx, gy, gz, gs = lat.download_f64()
    for got, want in zip((gx, gy, gz), cur):
        # the gradient tolerance above (2e-5) times eta, plus FP32 rounding
        np.testing.assert_allclose(got, want, rtol=0, atol=2e-6)
    assert np.array_equal(gs, s)
    lat.close()
