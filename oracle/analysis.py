"""Test infrastructure only: numpy restatements of the reference's analysis
functions, used by the tests as the checker of chllmodel_b200.analysis.
Nothing in the library imports this module.

- shell_corr: calc_n_corr and calc_s_corr of notebooks/paper_plots2.ipynb
  (cell 0, lines 61-112).  The reference loops over sites and offsets; here
  each offset d (|d|^2 < R^2) is one vectorised sum over the overlapping
  slices x, x + d (open boundaries) or over a rolled copy (periodic images),
  with the same per-pair terms: (n_x . n_y)^2 and s_x s_y - <s>^2, summed
  into shell floor(|d|) and divided by the shell's pair count.
- structure_factor: structure_factor / get_sc of
  notebooks/.ipynb_checkpoints/hero_stripe-checkpoint.py (lines 10-29): the
  direct sum of s_x exp(-i (kv p) . (x+1)) / N over all sites for every kv.
"""
from __future__ import annotations

import numpy as np


def _overlap(d: int, n: int):
    """Index ranges of x and x + d that both lie in [0, n)."""
    lo = max(0, -d)
    hi = n - max(0, d)
    return slice(lo, hi), slice(lo + d, hi + d)


def shell_corr(nx, ny, nz, s, nshells: int, wrap: bool = False):
    """(gn, gs, counts) of calc_n_corr / calc_s_corr (paper_plots2.ipynb cell 0,
    lines 61-112); wrap=True pairs x with the periodic image of x + d."""
    nx, ny, nz = (np.asarray(a, np.float64) for a in (nx, ny, nz))
    s = np.asarray(s, np.float64)
    ni, nj, nk = nx.shape
    R = int(nshells)
    gn = np.zeros(R)
    gs = np.zeros(R)
    c = np.zeros(R)
    s_avg2 = np.mean(s) ** 2
    for di in range(-R + 1, R):
        for dj in range(-R + 1, R):
            for dk in range(-R + 1, R):
                r2 = di * di + dj * dj + dk * dk
                if r2 >= R * R:
                    continue
                shell = int(np.floor(np.sqrt(r2)))
                if wrap:
                    sh = (-di, -dj, -dk)
                    ax, ay, az, as_ = nx, ny, nz, s
                    bx, by, bz, bs = (np.roll(a, sh, axis=(0, 1, 2)) for a in (nx, ny, nz, s))
                else:
                    (xi, yi), (xj, yj), (xk, yk) = _overlap(di, ni), _overlap(dj, nj), \
                        _overlap(dk, nk)
                    if xi.stop <= xi.start or xj.stop <= xj.start or xk.stop <= xk.start:
                        continue
                    ax, ay, az, as_ = (a[xi, xj, xk] for a in (nx, ny, nz, s))
                    bx, by, bz, bs = (a[yi, yj, yk] for a in (nx, ny, nz, s))
                dot = ax * bx + ay * by + az * bz
                gn[shell] += np.sum(dot * dot)
                gs[shell] += np.sum(as_ * bs - s_avg2)
                c[shell] += ax.size
    with np.errstate(invalid="ignore", divide="ignore"):
        return gn / c, gs / c, c


def structure_factor(s, bins: int, k_min: float, k_max: float, plane):
    """(sf, kvs) of hero_stripe's structure_factor: direct sum over all sites."""
    s = np.asarray(s, np.float64)
    ni, nj, nk = s.shape
    n3 = ni * nj * nk
    i, j, k = np.meshgrid(np.arange(1, ni + 1), np.arange(1, nj + 1), np.arange(1, nk + 1),
                          indexing="ij")
    kvs = np.linspace(k_min, k_max, bins)
    p = np.asarray(plane, np.float64)
    sc = np.empty(len(kvs), dtype=complex)
    for idx, kv in enumerate(kvs):
        kvec = kv * p
        phase = kvec[0] * i + kvec[1] * j + kvec[2] * k
        sc[idx] = np.sum(s * np.exp(-1j * phase)) / n3
    return sc.real * sc.real + sc.imag * sc.imag, kvs
