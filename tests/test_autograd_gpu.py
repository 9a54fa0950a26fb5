"""GPU tests of the torch.autograd.Function over the energy adjoint, the
coupling sensitivities and the zero-temperature gradient quench (the
differentiation workload: 64^3, 500 sweeps at kT = 0.3, K = 1, h = 0.5,
seed 3, then a 2000-step quench)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(shape, seed, sweeps=0, kT=0.3, K=1.0, h=0.5, boundary="periodic"):
    import torch

    from chllmodel_b200.lattice import Lattice, coupling

    lat = Lattice(*shape, boundary=boundary)
    lat.init_random(seed)
    lat.set_control(0.1, step=1)
    if sweeps:
        lat.sweep(coupling(kT, K, h), sweeps, seed=seed)
    f4 = torch.from_numpy(lat.download_f4()).cuda()
    return lat, f4[:, :3].contiguous(), f4[:, 3].contiguous()


def test_autograd_matches_fp64_oracle(oracle):
    import torch

    from chllmodel_b200.autograd import lattice_energy

    shape = (12, 10, 8)
    lat, n, s = _state(shape, 5, sweeps=10)
    n = n.clone().requires_grad_(True)
    eps = torch.tensor(1.1, dtype=torch.float64, requires_grad=True)
    K = torch.tensor(0.9, dtype=torch.float64, requires_grad=True)
    h = torch.tensor(0.3, dtype=torch.float64, requires_grad=True)
    E = lattice_energy(n, s, eps, K, h, shape)
    E.backward()
    nx, ny, nz, si = lat.download_f64()
    cfg = oracle.make_cfg(*shape, periodic=True, K=0.9, g=0.3, eps=1.1)
    og, out4 = oracle.energy_grad(cfg, nx, ny, nz, si)
    og = np.stack([og[..., c].ravel(order="F") for c in range(3)], 1)
    assert float(E) == pytest.approx(out4[0], rel=1e-9)
    np.testing.assert_allclose(n.grad.cpu().numpy(), og, rtol=2e-5, atol=2e-5)
    assert float(eps.grad) == pytest.approx(out4[1], rel=1e-9)
    assert float(K.grad) == pytest.approx(out4[2], rel=1e-9)
    assert float(h.grad) == pytest.approx(out4[3], rel=1e-9)
    lat.close()


def test_autograd_central_differences():
    """Central differences of the autograd energy itself (step 1e-3)."""
    import torch

    from chllmodel_b200.autograd import lattice_energy

    shape = (16, 16, 16)
    lat, n, s = _state(shape, 3, sweeps=20)
    n0 = n.clone().requires_grad_(True)
    E = lattice_energy(n0, s, 1.0, 1.0, 0.5, shape)
    E.backward()
    g = n0.grad
    rng = np.random.default_rng(1)
    for _ in range(40):
        x = int(rng.integers(0, n.shape[0]))
        c = int(rng.integers(0, 3))
        p, m = n.clone(), n.clone()
        p[x, c] += 1e-3
        m[x, c] -= 1e-3
        delta = float(p[x, c] - m[x, c])  # exact FP32 step
        fd = (float(lattice_energy(p, s, 1.0, 1.0, 0.5, shape)) -
              float(lattice_energy(m, s, 1.0, 1.0, 0.5, shape))) / delta
        assert float(g[x, c]) == pytest.approx(fd, abs=2e-4, rel=1e-3)
    lat.close()


def test_coupling_sensitivities_are_energy_derivatives():
    from chllmodel_b200.autograd import coupling_sensitivities

    shape = (16, 16, 16)
    lat, n, s = _state(shape, 9, sweeps=5)
    base = coupling_sensitivities(n, s, 1.0, 1.0, 0.5, shape)
    hstep = 1e-4
    for name, kw in (("dE_deps", 0), ("dE_dK", 1), ("dE_dh", 2)):
        args_p = [1.0, 1.0, 0.5]
        args_m = [1.0, 1.0, 0.5]
        args_p[kw] += hstep
        args_m[kw] -= hstep
        ep = coupling_sensitivities(n, s, *args_p, shape)["E"]
        em = coupling_sensitivities(n, s, *args_m, shape)["E"]
        assert base[name] == pytest.approx((ep - em) / (2 * hstep), rel=1e-6, abs=1e-6)
    lat.close()


def test_gradient_quench_64cube():
    """500 sweeps at kT = 0.3 (seed 3), then 2000 quench steps at kT = 0:
    the energy never rises and the torque shrinks."""
    import torch

    from chllmodel_b200.autograd import quench, tangent_gradient

    shape = (64, 64, 64)
    lat, n, s = _state(shape, 3, sweeps=500)
    g0 = tangent_gradient(n, s, 1.0, 1.0, 0.5, shape)
    energies = quench(lat, eps=1.0, K=1.0, h=0.5, eta=0.05, nsteps=2000, report_every=100)
    es = [e for _, e in energies]
    assert len(es) == 20
    assert all(b <= a + 1e-6 * abs(a) for a, b in zip(es, es[1:]))
    f4 = torch.from_numpy(lat.download_f4()).cuda()
    g1 = tangent_gradient(f4[:, :3].contiguous(), f4[:, 3].contiguous(), 1.0, 1.0, 0.5, shape)
    assert float(g1.norm()) < 0.2 * float(g0.norm())
    # chiralities untouched, directors unit length
    assert torch.equal(f4[:, 3], s)
    assert float((f4[:, :3].norm(dim=1) - 1).abs().max()) < 1e-5
    lat.close()
