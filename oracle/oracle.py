"""TEST INFRASTRUCTURE ONLY -- ctypes binding of the CPU oracle.

The oracle (``chll_oracle.c``) restates the reference's checkerboard
Metropolis path (mdeutsc2/ChLLModel ``chll/chll_mod.f90``) in C with the same
Philox random stream as the CUDA library.  It is the checker of the parity
tests, of ``__graft_entry__.smoke()`` and the timed CPU baseline of
``bench.py``; the product never imports this module.

All arrays are natural F-order (``order='F'``, shape (ni, nj, nk)): FP64
directors and int32 chiralities, as in the reference's ``ChLLSim``
(chll/chll.py:57-61).
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_chll.so")
_lib = None


class Cfg(ct.Structure):
    """Mirror of ``oracle_cfg`` in chll_oracle.c."""

    _fields_ = [
        ("ni", ct.c_int), ("nj", ct.c_int), ("nk", ct.c_int), ("periodic", ct.c_int),
        ("kT", ct.c_double), ("K", ct.c_double), ("g", ct.c_double), ("eps", ct.c_double),
        ("seed", ct.c_uint64), ("replica", ct.c_uint32), ("pad", ct.c_int32),
    ]


def make_cfg(ni, nj, nk, *, periodic=False, kT=0.5, K=0.5, g=0.0, eps=1.0, seed=1, replica=0):
    return Cfg(ni, nj, nk, int(bool(periodic)), float(kT), float(K), float(g), float(eps),
               int(seed), int(replica), 0)


def build() -> str:
    """Compiles liboracle_chll.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = ct.CDLL(_LIB_PATH)
    d_arr = np.ctypeslib.ndpointer(dtype=np.float64, flags="F_CONTIGUOUS")
    i_arr = np.ctypeslib.ndpointer(dtype=np.int32, flags="F_CONTIGUOUS")
    P = ct.POINTER
    L.oracle_philox.argtypes = [P(ct.c_uint32), P(ct.c_uint32), P(ct.c_uint32)]
    L.oracle_philox.restype = None
    L.oracle_site_energy.argtypes = [P(Cfg), d_arr, d_arr, d_arr, i_arr, ct.c_int, ct.c_int,
                                     ct.c_int, ct.c_double, ct.c_double, ct.c_double, ct.c_int]
    L.oracle_site_energy.restype = ct.c_float
    L.oracle_propose.argtypes = [ct.c_double] * 5 + [P(ct.c_double)] * 3
    L.oracle_propose.restype = None
    L.oracle_pass.argtypes = [P(Cfg), ct.c_int, ct.c_uint32, ct.c_double, d_arr, d_arr, d_arr,
                              i_arr, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    L.oracle_pass.restype = ct.c_longlong
    L.oracle_etot.argtypes = [P(Cfg), d_arr, d_arr, d_arr, i_arr, ct.c_int, P(ct.c_double)]
    L.oracle_etot.restype = ct.c_float
    L.oracle_moments.argtypes = [P(Cfg), d_arr, d_arr, d_arr, i_arr, P(ct.c_double)]
    L.oracle_moments.restype = None
    L.oracle_run.argtypes = [P(Cfg), ct.c_int, ct.c_int, ct.c_int, ct.c_longlong,
                             P(ct.c_double), d_arr, d_arr, d_arr, i_arr, ct.c_void_p,
                             ct.c_void_p, ct.c_int]
    L.oracle_run.restype = ct.c_int
    L.oracle_chain.argtypes = [P(Cfg), ct.c_int, ct.c_int, ct.c_int, ct.c_longlong,
                               P(ct.c_double), d_arr, d_arr, d_arr, i_arr, ct.c_void_p]
    L.oracle_chain.restype = ct.c_int
    L.oracle_init_random.argtypes = [P(Cfg), d_arr, d_arr, d_arr, i_arr]
    L.oracle_init_random.restype = None
    L.oracle_energy_grad.argtypes = [P(Cfg), d_arr, d_arr, d_arr, i_arr, ct.c_void_p,
                                     ct.c_void_p, ct.c_void_p, ct.c_int, P(ct.c_double)]
    L.oracle_energy_grad.restype = None
    L.oracle_max_threads.argtypes = []
    L.oracle_max_threads.restype = ct.c_int
    L.oracle_set_threads.argtypes = [ct.c_int]
    L.oracle_set_threads.restype = None
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


def new_state(ni, nj, nk):
    z = lambda dt: np.zeros((ni, nj, nk), dtype=dt, order="F")
    return z(np.float64), z(np.float64), z(np.float64), z(np.int32)


def philox(ctr, key):
    c = (ct.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in ctr])
    k = (ct.c_uint32 * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    o = (ct.c_uint32 * 4)()
    lib().oracle_philox(c, k, o)
    return [int(x) for x in o]


def site_energy(cfg, nx, ny, nz, s, i, j, k, m=None, snew=None):
    if m is None:
        m = (nx[i, j, k], ny[i, j, k], nz[i, j, k])
    if snew is None:
        snew = int(s[i, j, k])
    return lib().oracle_site_energy(ct.byref(cfg), nx, ny, nz, s, i, j, k, float(m[0]),
                                    float(m[1]), float(m[2]), int(snew))


def propose(n, d, u):
    out = [ct.c_double(), ct.c_double(), ct.c_double()]
    lib().oracle_propose(float(n[0]), float(n[1]), float(n[2]), float(d), float(u),
                         *[ct.byref(o) for o in out])
    return np.array([o.value for o in out])


def run_pass(cfg, p, step, d, nx, ny, nz, s, detail=False):
    """One half-sweep in place.  With detail=True also returns per-site
    accept flags, enew-eold and the acceptance uniform (natural order)."""
    if detail:
        shape = nx.shape
        acc = np.full(shape, -1, dtype=np.int8, order="F")
        de = np.full(shape, np.nan, dtype=np.float64, order="F")
        u = np.full(shape, np.nan, dtype=np.float64, order="F")
        n = lib().oracle_pass(ct.byref(cfg), int(p), int(step) & 0xFFFFFFFF, float(d), nx, ny,
                              nz, s, _ptr(acc), _ptr(de), _ptr(u))
        return n, acc, de, u
    return lib().oracle_pass(ct.byref(cfg), int(p), int(step) & 0xFFFFFFFF, float(d), nx, ny, nz,
                             s, None, None, None)


def etot(cfg, nx, ny, nz, s, mode=0):
    """Returns (FP32 per-site value, FP64 sum) of chll_mod.f90:414-456
    (mode 0) or of the lattice-boundary total energy (mode 1)."""
    tot = ct.c_double()
    v = lib().oracle_etot(ct.byref(cfg), nx, ny, nz, s, int(mode), ct.byref(tot))
    return float(v), tot.value


def moments(cfg, nx, ny, nz, s):
    out = (ct.c_double * 9)()
    lib().oracle_moments(ct.byref(cfg), nx, ny, nz, s, out)
    return np.array(list(out))


def run(cfg, nstart, nstop, nout, d, nx, ny, nz, s, adapt_until=10000):
    rows = (1 + nstop - nstart) // nout
    msteps = np.zeros(max(rows, 1), dtype=np.int32)
    m = np.zeros((max(rows, 1), 5), dtype=np.float64, order="F")
    dd = ct.c_double(d)
    nmeas = lib().oracle_run(ct.byref(cfg), nstart, nstop, nout, int(adapt_until), ct.byref(dd),
                             nx, ny, nz, s, _ptr(msteps), _ptr(m), rows)
    return msteps[:rows], m[:rows], dd.value, nmeas


def chain(cfg, burn, nmeas, every, d, nx, ny, nz, s, adapt_until=10000):
    """An equilibrium chain from step 1 (the reference step loop with its d
    rule): returns (nmeas x 9 FP64 moments after sweep burn, every `every`
    sweeps, as moments() gives them; the final d)."""
    out = np.zeros((nmeas, 9), np.float64)
    dd = ct.c_double(d)
    got = lib().oracle_chain(ct.byref(cfg), int(burn), int(nmeas), int(every), int(adapt_until),
                             ct.byref(dd), nx, ny, nz, s, _ptr(out))
    return out[:got], dd.value


def init_random(cfg):
    nx, ny, nz, s = new_state(cfg.ni, cfg.nj, cfg.nk)
    lib().oracle_init_random(ct.byref(cfg), nx, ny, nz, s)
    return nx, ny, nz, s


def energy_grad(cfg, nx, ny, nz, s, project=False):
    gx, gy, gz, _ = new_state(cfg.ni, cfg.nj, cfg.nk)
    out = (ct.c_double * 4)()
    lib().oracle_energy_grad(ct.byref(cfg), nx, ny, nz, s, _ptr(gx), _ptr(gy), _ptr(gz),
                             int(bool(project)), out)
    return np.stack([gx, gy, gz], axis=-1), np.array(list(out))


def set_threads(n):
    lib().oracle_set_threads(int(n))


def max_threads():
    return lib().oracle_max_threads()
