"""Device-resident red/black lattice: the handle API of libchll_mod.so.

A ``Lattice`` owns one float4 (nx, ny, nz, s) lattice on the current CUDA
device, split by checkerboard colour, plus its device control block (d, step,
accept fractions).  It is what ``ChLLSim.run`` uses underneath, and what the
bench, the lockstep parity tests and the autograd wrapper drive directly.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib
from ._lib import Coupling, check


def coupling(kT: float, K: float, g: float = 0.0, eps: float = 1.0) -> Coupling:
    return Coupling(float(kT), float(K), float(g), float(eps))


# chll_lattice_pass codes of the fused sweep's passes
FUSED_A0, FUSED_A, FUSED_B, FUSED_F = 4, 5, 6, 7


class Lattice:
    """One ni x nj x nk lattice on the GPU (boundary 'open' or 'periodic')."""

    def __init__(self, ni: int, nj: int, nk: int, boundary: str = "open"):
        if boundary not in ("open", "periodic"):
            raise ValueError("boundary must be 'open' or 'periodic'")
        self._L = _lib.load()
        self.ni, self.nj, self.nk = int(ni), int(nj), int(nk)
        self.boundary = boundary
        h = ct.c_void_p()
        check(self._L.chll_lattice_create(self.ni, self.nj, self.nk,
                                          _lib.CHLL_PERIODIC if boundary == "periodic"
                                          else _lib.CHLL_OPEN, ct.byref(h)))
        self._h = h

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.chll_lattice_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> ct.c_void_p:
        return self._h

    @property
    def nsites(self) -> int:
        return self.ni * self.nj * self.nk

    # -- state ------------------------------------------------------------
    def set_stream(self, stream_ptr: int | None) -> None:
        check(self._L.chll_lattice_set_stream(self._h, ct.c_void_p(stream_ptr or 0)))

    def set_kernel(self, kind: str) -> None:
        """Sweep form: 'auto' ('resident' up to about 32^3, else 'fused'),
        'fused' (two passes per sweep),
        'direct' (the reference's four half-sweeps, neighbours from global
        memory), 'staged' (four half-sweeps from shared-memory row tiles) or
        'resident' (the fused passes of a whole chunk in one thread-block
        cluster launch, for small lattices).  All give the same chain bit for
        bit."""
        code = {"auto": 0, "direct": 1, "staged": 2, "fused": 3, "resident": 4}[kind]
        check(self._L.chll_lattice_set_kernel(self._h, code))

    def sync(self) -> None:
        check(self._L.chll_lattice_sync(self._h))

    def init_random(self, seed: int, replica: int = 0) -> None:
        check(self._L.chll_lattice_init_random(self._h, int(seed), int(replica)))

    def upload_f64(self, nx, ny, nz, s) -> None:
        arrs = [np.asfortranarray(nx, dtype=np.float64), np.asfortranarray(ny, dtype=np.float64),
                np.asfortranarray(nz, dtype=np.float64), np.asfortranarray(s, dtype=np.int32)]
        for a in arrs:
            if a.size != self.nsites:
                raise ValueError("array size does not match the lattice")
        check(self._L.chll_lattice_upload_f64(self._h, *[a.ctypes.data_as(ct.c_void_p)
                                                          for a in arrs]))

    def download_f64(self):
        shape = (self.ni, self.nj, self.nk)
        nx, ny, nz = (np.zeros(shape, np.float64, order="F") for _ in range(3))
        s = np.zeros(shape, np.int32, order="F")
        check(self._L.chll_lattice_download_f64(self._h, *[a.ctypes.data_as(ct.c_void_p)
                                                            for a in (nx, ny, nz, s)]))
        return nx, ny, nz, s

    def upload_f4(self, xyzs) -> None:
        """Natural-order float4 records: a host array (N,4) or a device pointer."""
        if isinstance(xyzs, int):
            check(self._L.chll_lattice_upload_f4(self._h, ct.c_void_p(xyzs)))
            return
        a = np.ascontiguousarray(xyzs, dtype=np.float32).reshape(-1, 4)
        if a.shape[0] != self.nsites:
            raise ValueError("array size does not match the lattice")
        check(self._L.chll_lattice_upload_f4(self._h, a.ctypes.data_as(ct.c_void_p)))

    def download_f4(self, out_ptr: int | None = None):
        if out_ptr is not None:
            check(self._L.chll_lattice_download_f4(self._h, ct.c_void_p(out_ptr)))
            return None
        a = np.zeros((self.nsites, 4), np.float32)
        check(self._L.chll_lattice_download_f4(self._h, a.ctypes.data_as(ct.c_void_p)))
        return a

    def storage(self):
        """(colour0 device ptr, colour1 device ptr, float4 per colour, hx)."""
        c0, c1, n, hx = ct.c_void_p(), ct.c_void_p(), ct.c_int64(), ct.c_int32()
        check(self._L.chll_lattice_storage(self._h, ct.byref(c0), ct.byref(c1), ct.byref(n),
                                           ct.byref(hx)))
        return c0.value, c1.value, n.value, hx.value

    # -- control ----------------------------------------------------------
    def set_control(self, d: float, step: int = 1, adapt_until: int = 10000) -> None:
        check(self._L.chll_lattice_set_control(self._h, float(d), int(step), int(adapt_until)))

    def control(self) -> dict:
        d, st, pa, fa = ct.c_double(), ct.c_int64(), ct.c_double(), ct.c_double()
        check(self._L.chll_lattice_get_control(self._h, ct.byref(d), ct.byref(st), ct.byref(pa),
                                               ct.byref(fa)))
        return {"d": d.value, "step": st.value, "paccept": pa.value, "faccept": fa.value}

    # -- compute ----------------------------------------------------------
    def sweep(self, cp: Coupling, nsweeps: int, seed: int = 1, replica: int = 0) -> None:
        check(self._L.chll_lattice_sweep(self._h, ct.byref(cp), int(seed), int(replica),
                                         int(nsweeps)))

    def half_sweep(self, cp: Coupling, p: int, seed: int = 1, replica: int = 0) -> None:
        """One pass: 0-3 the reference's half-sweeps (director colour 0/1,
        chirality colour 0/1); FUSED_A0 / FUSED_A / FUSED_B / FUSED_F the
        fused sweep's passes (steps: A0 B (A B)... F)."""
        check(self._L.chll_lattice_pass(self._h, ct.byref(cp), int(seed), int(replica), int(p)))

    def reserve_rows(self, n: int) -> None:
        check(self._L.chll_lattice_reserve_rows(self._h, int(n)))

    def measure(self, cp: Coupling, slot: int) -> None:
        """Enqueues the FP64 observables into device row `slot` (no wait)."""
        check(self._L.chll_lattice_measure(self._h, ct.byref(cp), int(slot)))

    def read_rows(self, first: int, count: int) -> np.ndarray:
        rows = np.zeros((count, _lib.ROW_LEN), np.float64)
        check(self._L.chll_lattice_read_rows(self._h, rows.ctypes.data_as(ct.c_void_p),
                                             int(first), int(count)))
        return rows

    def observe(self, cp: Coupling) -> np.ndarray:
        row = np.zeros(_lib.ROW_LEN, np.float64)
        check(self._L.chll_lattice_observe(self._h, ct.byref(cp),
                                           row.ctypes.data_as(ct.c_void_p)))
        return row

    def quench(self, cp: Coupling, eta: float, nsteps: int) -> None:
        """nsteps of zero-temperature tangent gradient descent (asynchronous)."""
        check(self._L.chll_lattice_quench(self._h, ct.byref(cp), float(eta), int(nsteps)))

    def energy_grad(self, cp: Coupling, project: bool = False, grad_ptr: int | None = None):
        """Returns (grad (N,4) host array or None if grad_ptr given, out4)."""
        out4 = np.zeros(4, np.float64)
        if grad_ptr is not None:
            check(self._L.chll_lattice_energy_grad(self._h, ct.byref(cp), ct.c_void_p(grad_ptr),
                                                   int(bool(project)),
                                                   out4.ctypes.data_as(ct.c_void_p)))
            return None, out4
        g = np.zeros((self.nsites, 4), np.float32)
        check(self._L.chll_lattice_energy_grad(self._h, ct.byref(cp),
                                               g.ctypes.data_as(ct.c_void_p), int(bool(project)),
                                               out4.ctypes.data_as(ct.c_void_p)))
        return g, out4


def to_f4(nx, ny, nz, s) -> np.ndarray:
    """F-order arrays -> natural-order (N,4) float32 records."""
    return np.stack([np.ravel(nx, order="F"), np.ravel(ny, order="F"), np.ravel(nz, order="F"),
                     np.ravel(s, order="F")], axis=1).astype(np.float32)


def from_f4(a, ni, nj, nk):
    """Natural-order (N,4) records -> F-order FP64 nx, ny, nz and int32 s."""
    a = np.asarray(a).reshape(-1, 4)
    shp = (ni, nj, nk)
    f = lambda col, dt: np.asfortranarray(a[:, col].astype(dt).reshape(shp, order="F"))
    return f(0, np.float64), f(1, np.float64), f(2, np.float64), f(3, np.int32)
