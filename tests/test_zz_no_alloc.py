"""The no-allocation energy adjoint, chll_energy_grad_noalloc, called through
the C ABI, against the allocating chll_lattice_energy_grad.

It exists for callers that cannot let a library call cudaMalloc -- a
Fortran/OpenACC host whose arrays live in its runtime's device pool, or an
application whose own allocator holds nearly all of HBM -- so it keeps every
intermediate in one fixed device array of the library.  This file is
collected last: two calls in a row must each reproduce the allocating entry
point, and a lattice larger than the fixed array must be refused."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRAD_RTOL = 2e-5   # the adjoint tests' tolerance for the FP32 gradient
GRAD_ATOL = 2e-5
SUM_RTOL = 1e-9    # and for the FP64 sums


@pytest.mark.parametrize("shape,boundary", [((64, 64, 64), "periodic"),
                                            ((37, 20, 12), "open")])
def test_noalloc_adjoint_matches_allocating_entry_point(shape, boundary):
    import torch

    from chllmodel_b200 import _lib
    from chllmodel_b200.lattice import Lattice, coupling

    L = _lib.load()
    lat = Lattice(*shape, boundary=boundary)
    lat.init_random(seed=5)
    cp = coupling(0.3, 1.0, 0.5, 1.1)
    lat.set_control(0.1, step=1)
    lat.sweep(cp, 4, seed=5)
    ref_grad, ref_out4 = lat.energy_grad(cp, project=True)   # allocating entry point
    c0, c1, _, _ = lat.storage()
    n = lat.nsites
    grad = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    out4 = torch.empty(4, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    bnd = _lib.CHLL_PERIODIC if boundary == "periodic" else _lib.CHLL_OPEN
    for _ in range(2):
        grad.fill_(float("nan"))
        out4.fill_(float("nan"))
        rc = L.chll_energy_grad_noalloc(ct.c_void_p(c0), ct.c_void_p(c1), *shape, bnd,
                                        ct.byref(cp), 1, ct.c_void_p(grad.data_ptr()),
                                        ct.c_void_p(out4.data_ptr()), ct.c_void_p(stream))
        _lib.check(rc)
        torch.cuda.synchronize()
        np.testing.assert_allclose(grad.cpu().numpy(), ref_grad, rtol=GRAD_RTOL, atol=GRAD_ATOL)
        np.testing.assert_allclose(out4.cpu().numpy(), ref_out4, rtol=SUM_RTOL, atol=SUM_RTOL)
    lat.close()


def test_noalloc_adjoint_refuses_lattices_beyond_its_scratch():
    import torch

    from chllmodel_b200 import _lib
    from chllmodel_b200.lattice import Lattice, coupling

    L = _lib.load()
    lat = Lattice(66, 64, 64, boundary="periodic")   # 2*34*64*64 slots > 262,144
    c0, c1, _, _ = lat.storage()
    out4 = torch.empty(4, dtype=torch.float64, device="cuda")
    rc = L.chll_energy_grad_noalloc(ct.c_void_p(c0), ct.c_void_p(c1), 66, 64, 64,
                                    _lib.CHLL_PERIODIC, ct.byref(coupling(0.3, 1.0)), 0, None,
                                    ct.c_void_p(out4.data_ptr()), None)
    assert rc == _lib.CHLL_ERANGE
    assert "at most 262144" in _lib.last_error()
    lat.close()


def test_noalloc_adjoint_on_16_byte_aligned_arrays():
    """Caller arrays that start 16 but not 32 bytes aligned (a float4 array
    at an odd slot) take the one-slot-per-thread kernel, with the same
    results as the library's own 32-byte aligned storage."""
    import torch

    from chllmodel_b200 import _lib
    from chllmodel_b200.lattice import Lattice, coupling

    L = _lib.load()
    shape = (20, 18, 10)
    lat = Lattice(*shape, boundary="periodic")
    lat.init_random(seed=8)
    cp = coupling(0.3, 1.0, 0.5, 1.1)
    lat.set_control(0.1, step=1)
    lat.sweep(cp, 3, seed=8)
    ref_grad, ref_out4 = lat.energy_grad(cp, project=True)
    c0, c1, per_colour, _ = lat.storage()
    # copies of both colour arrays one float4 past a 256-byte aligned start
    buf = torch.empty((2, per_colour + 2, 4), dtype=torch.float32, device="cuda")
    for c, src in enumerate((c0, c1)):
        view = torch.as_tensor(_DeviceF4(src, per_colour), device="cuda")
        buf[c, 1:per_colour + 1].copy_(view)
    p0, p1 = buf[0, 1:].data_ptr(), buf[1, 1:].data_ptr()
    assert p0 % 32 == 16 and p1 % 32 == 16
    n = lat.nsites
    grad = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    out4 = torch.empty(4, dtype=torch.float64, device="cuda")
    rc = L.chll_energy_grad_noalloc(ct.c_void_p(p0), ct.c_void_p(p1), *shape, _lib.CHLL_PERIODIC,
                                    ct.byref(cp), 1, ct.c_void_p(grad.data_ptr()),
                                    ct.c_void_p(out4.data_ptr()),
                                    ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc)
    torch.cuda.synchronize()
    np.testing.assert_allclose(grad.cpu().numpy(), ref_grad, rtol=GRAD_RTOL, atol=GRAD_ATOL)
    np.testing.assert_allclose(out4.cpu().numpy(), ref_out4, rtol=SUM_RTOL, atol=SUM_RTOL)
    lat.close()


def test_noalloc_adjoint_refuses_misaligned_arrays():
    """Arrays that are not float4 (16-byte) aligned, or an out4 that is not
    8-byte aligned, are refused on the host before any launch: a kernel
    given them would fault on its vector accesses and lose the context."""
    import torch

    from chllmodel_b200 import _lib
    from chllmodel_b200.lattice import Lattice, coupling

    L = _lib.load()
    shape = (16, 12, 8)
    lat = Lattice(*shape, boundary="periodic")
    lat.init_random(seed=2)
    c0, c1, _, _ = lat.storage()
    n = lat.nsites
    buf = torch.zeros(4 * n + 8, dtype=torch.float32, device="cuda")
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    grad = buf.data_ptr()
    out4 = out.data_ptr()
    cp = coupling(0.3, 1.0)
    args = dict(c0=c0, c1=c1, grad=grad, out4=out4)
    for key, off in (("c0", 8), ("c1", 4), ("grad", 8), ("out4", 4)):
        a = dict(args)
        a[key] += off
        rc = L.chll_energy_grad_noalloc(ct.c_void_p(a["c0"]), ct.c_void_p(a["c1"]), *shape,
                                        _lib.CHLL_PERIODIC, ct.byref(cp), 1,
                                        ct.c_void_p(a["grad"]), ct.c_void_p(a["out4"]), None)
        assert rc == _lib.CHLL_EINVAL, key
        assert "aligned" in _lib.last_error()
    # the same call with aligned arrays runs
    rc = L.chll_energy_grad_noalloc(ct.c_void_p(c0), ct.c_void_p(c1), *shape, _lib.CHLL_PERIODIC,
                                    ct.byref(cp), 1, ct.c_void_p(grad), ct.c_void_p(out4), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    assert torch.isfinite(out[:4]).all()
    lat.close()


class _DeviceF4:
    """(count, 4) float32 device array at an address, for torch.as_tensor."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (count, 4), "typestr": "<f4",
                                         "data": (ptr, False), "version": 3, "strides": None}
