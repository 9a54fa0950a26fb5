"""``torch.autograd.Function`` over the hand-written energy adjoint kernel.

``lattice_energy(n, s, eps, K, h, shape, boundary)`` returns the FP64 total
energy of a lattice whose directors ``n`` (N x 3, FP32, CUDA, natural order
i fastest) and chiralities ``s`` (N, +-1) are torch tensors; its backward
pass comes from the adjoint kernel (``energy_grad_unit_kernel``: dE/dn for every site, plus
dE/deps, dE/dK, dE/dh in FP64), not from autograd tracing.  The Metropolis
sweep itself is not differentiated: acceptance stays exactly the reference's
rule (chll_mod.f90:188-200).

``quench`` runs the zero-temperature gradient descent on the device, and
``coupling_sensitivities`` returns dE/d(eps, K, h) of a lattice state.
This module is the only place the package uses torch on the compute side.
"""
from __future__ import annotations

import torch

from . import _lib
from .lattice import Lattice, coupling

_cache: dict = {}


def _lattice(shape, boundary, device) -> Lattice:
    key = (tuple(int(x) for x in shape), boundary, int(device))
    lat = _cache.get(key)
    if lat is None:
        with torch.cuda.device(device):
            lat = Lattice(*key[0], boundary=boundary)
        _cache[key] = lat
    return lat


def _stream_handle() -> int:
    return _lib.torch_stream_handle()


def _pack(n: torch.Tensor, s: torch.Tensor) -> torch.Tensor:
    return torch.cat([n.detach().to(torch.float32), s.detach().to(torch.float32).reshape(-1, 1)],
                     dim=1).contiguous()


class LatticeEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, n, s, eps, K, h, shape, boundary):
        if not n.is_cuda:
            raise ValueError("lattice_energy needs CUDA tensors (the kernels have no CPU path)")
        N = int(shape[0]) * int(shape[1]) * int(shape[2])
        if n.shape != (N, 3) or s.numel() != N:
            raise ValueError(f"n must be ({N}, 3) and s ({N},) for lattice {tuple(shape)}")
        lat = _lattice(shape, boundary, n.device.index or 0)
        lat.set_stream(_stream_handle())
        packed = _pack(n, s)
        lat.upload_f4(packed.data_ptr())
        grad = torch.empty((N, 4), dtype=torch.float32, device=n.device)
        cp = coupling(0.0, float(K), float(h), float(eps))
        _, out4 = lat.energy_grad(cp, project=False, grad_ptr=grad.data_ptr())
        dev = n.device
        ctx.save_for_backward(grad[:, :3].to(n.dtype),
                              torch.tensor(out4[1:], dtype=torch.float64, device=dev))
        return torch.tensor(out4[0], dtype=torch.float64, device=dev)

    @staticmethod
    def backward(ctx, g_out):
        grad_n, d_couplings = ctx.saved_tensors
        g = g_out.to(torch.float64)
        gn = (g.to(grad_n.dtype) * grad_n) if ctx.needs_input_grad[0] else None
        ge = g * d_couplings[0] if ctx.needs_input_grad[2] else None
        gk = g * d_couplings[1] if ctx.needs_input_grad[3] else None
        gh = g * d_couplings[2] if ctx.needs_input_grad[4] else None
        return gn, None, ge, gk, gh, None, None


def lattice_energy(n, s, eps, K, h, shape, boundary="periodic"):
    """Total energy (FP64) with analytic gradients to n, eps, K and h.

    eps, K, h may be python floats or 0-d tensors (requires_grad for their
    derivatives)."""
    as_t = lambda v: v if torch.is_tensor(v) else torch.tensor(float(v), dtype=torch.float64)
    return LatticeEnergy.apply(n, s, as_t(eps), as_t(K), as_t(h), tuple(shape), boundary)


def tangent_gradient(n, s, eps, K, h, shape, boundary="periodic") -> torch.Tensor:
    """(I - n n^T) dE/dn: the torque direction on every director."""
    N = n.shape[0]
    lat = _lattice(shape, boundary, n.device.index or 0)
    lat.set_stream(_stream_handle())
    lat.upload_f4(_pack(n, s).data_ptr())
    grad = torch.empty((N, 4), dtype=torch.float32, device=n.device)
    lat.energy_grad(coupling(0.0, float(K), float(h), float(eps)), project=True,
                    grad_ptr=grad.data_ptr())
    return grad[:, :3]


def coupling_sensitivities(n, s, eps, K, h, shape, boundary="periodic") -> dict:
    """E and dE/d(eps, K, h) of a lattice state, FP64."""
    lat = _lattice(shape, boundary, n.device.index or 0)
    lat.set_stream(_stream_handle())
    lat.upload_f4(_pack(n, s).data_ptr())
    _, out4 = lat.energy_grad(coupling(0.0, float(K), float(h), float(eps)))
    return {"E": out4[0], "dE_deps": out4[1], "dE_dK": out4[2], "dE_dh": out4[3]}


def quench(lat: Lattice, eps: float, K: float, h: float, eta: float, nsteps: int,
           report_every: int = 0):
    """Zero-temperature gradient quench of a device lattice: nsteps of
    n <- normalise(n - eta (I - n n^T) dE/dn), colour by colour.  Returns the
    FP64 energies after every `report_every` steps (and at the end)."""
    cp = coupling(0.0, K, h, eps)
    energies = []
    done = 0
    chunk = report_every if report_every > 0 else nsteps
    while done < nsteps:
        step = min(chunk, nsteps - done)
        lat.quench(cp, eta, step)
        done += step
        _, out4 = lat.energy_grad(cp)
        energies.append((done, out4[0]))
    return energies
