"""Analyses of a lattice's state on the device.

The reference computes these in numba on saved configurations:

- ``shell_correlations`` -- calc_n_corr and calc_s_corr of
  notebooks/paper_plots2.ipynb (cell 0, lines 61-112): shell-averaged nematic
  correlation <(n_x . n_y)^2> and chirality correlation <s_x s_y> - <s>^2 over
  all ordered pairs with |x - y| < nshells, shell floor(|x - y|), open
  boundaries (``wrap=True`` takes periodic images instead);
- ``structure_factor`` -- structure_factor / get_sc of
  notebooks/.ipynb_checkpoints/hero_stripe-checkpoint.py (lines 10-29):
  |sum_x s_x exp(-i kv p.(x+1)) / N|^2 for kv on a grid and an integer
  direction p.  Here the sum over sites is first binned on the device by the
  integer m = p.(x+1) (exact integer sums), and the transform over the few
  thousand bins runs on the host in FP64.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib
from ._lib import check
from .lattice import Lattice


def shell_correlations(lat: Lattice, nshells: int, wrap: bool = False):
    """Returns (gn, gs, counts), each of nshells FP64 values, as calc_n_corr's g,
    calc_s_corr's g and their common c."""
    L = _lib.load()
    gn = np.zeros(nshells, np.float64)
    gs = np.zeros(nshells, np.float64)
    cnt = np.zeros(nshells, np.float64)
    check(L.chll_lattice_shell_corr(lat._h, int(nshells), int(bool(wrap)),
                                    gn.ctypes.data_as(ct.c_void_p),
                                    gs.ctypes.data_as(ct.c_void_p),
                                    cnt.ctypes.data_as(ct.c_void_p)))
    return gn, gs, cnt


def projection(lat: Lattice, plane):
    """(m, hist): hist[t] = sum of s over sites with p.(i+1, j+1, k+1) = m[t]."""
    L = _lib.load()
    p = (ct.c_int * 3)(*[int(v) for v in plane])
    m0, nb = ct.c_longlong(), ct.c_int32()
    check(L.chll_lattice_projection(lat._h, p, None, ct.byref(m0), ct.byref(nb)))
    hist = np.zeros(nb.value, np.int64)
    check(L.chll_lattice_projection(lat._h, p, hist.ctypes.data_as(ct.c_void_p), ct.byref(m0),
                                    ct.byref(nb)))
    return m0.value + np.arange(nb.value, dtype=np.int64), hist


def structure_factor(lat: Lattice, bins: int, k_min: float, k_max: float, plane):
    """(sf, kvs) as hero_stripe's structure_factor(s, bins, k_min, k_max, plane)."""
    m, hist = projection(lat, plane)
    kvs = np.linspace(k_min, k_max, bins)
    n3 = lat.ni * lat.nj * lat.nk
    keep = hist != 0
    mm, hh = m[keep].astype(np.float64), hist[keep].astype(np.float64)
    sc = np.empty(len(kvs), dtype=complex)
    for idx, kv in enumerate(kvs):
        sc[idx] = np.sum(hh * np.exp(-1j * kv * mm)) / n3
    sf = sc.real * sc.real + sc.imag * sc.imag
    return sf, kvs
