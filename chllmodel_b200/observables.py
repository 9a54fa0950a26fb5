"""Derived observables from the FP64 moments the device accumulates.

The reference computes these only in its analysis notebooks:
  * specific heat, C_v = (<E^2> - <E>^2)/kT on the per-site energy column of
    the measurement rows (notebooks/paper_plots2.ipynb cell 0,
    calc_specific_heat; Xch-checkpoint cell 2);
  * chiral susceptibility, chi_c = N*(<eta^2> - <eta>^2)/kT
    (paper_plots-checkpoint cell 8), or without the N/kT factor
    (Xch-checkpoint cell 2).
Both reference forms are provided next to the standard fluctuation formulas
C_v = N*var(e)/kT^2 and chi = N*var(eta)/kT.  The nematic order parameter S
(largest eigenvalue of Q = (3/2)<n n^T> - I/2) does not exist in the
reference; it is defined here and computed from the Q-tensor raw moments.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib

# chll_batch_moments columns
B_NMEAS, B_SUM_E, B_SUM_E2, B_SUM_ETA, B_SUM_ETA2, B_SUM_ABS_ETA, B_SUM_S, B_SUM_S2 = range(8)
B_LAST_E, B_LAST_ETA, B_LAST_S, B_D, B_STEP, B_PACCEPT, B_FACCEPT, B_STATUS = range(8, 16)


def q_tensor(sums6, n):
    """Q = (3/2)<n n^T> - I/2 from the raw sums (xx, yy, zz, xy, xz, yz)."""
    xx, yy, zz, xy, xz, yz = (float(v) / n for v in sums6)
    q = 1.5 * np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]]) - 0.5 * np.eye(3)
    return q


def nematic_S(sums6, n) -> float:
    """Largest eigenvalue of Q (FP64)."""
    return float(np.linalg.eigvalsh(q_tensor(sums6, n))[-1])


def specific_heat_reference(e_rows, kT) -> float:
    """(<E^2> - <E>^2)/kT on per-site energies, as the notebooks compute it."""
    e = np.asarray(e_rows, dtype=np.float64)
    return float((np.mean(e * e) - np.mean(e) ** 2) / kT)


def specific_heat(e_per_site, kT, n) -> float:
    """Standard C_v per site: N*var(e)/kT^2."""
    e = np.asarray(e_per_site, dtype=np.float64)
    return float(n * (np.mean(e * e) - np.mean(e) ** 2) / (kT * kT))


def chiral_susceptibility(eta, kT, n, reference_form=True) -> float:
    """N*(<eta^2> - <eta>^2)/kT (paper_plots-checkpoint cell 8); with
    reference_form=False the bare variance of Xch-checkpoint cell 2."""
    x = np.asarray(eta, dtype=np.float64)
    var = np.mean(x * x) - np.mean(x) ** 2
    return float(n * var / kT) if reference_form else float(var)


def summarize_rows(rows16, kT, tail=None) -> dict:
    """Observables from ChLLSim.rows (one CHLL_ROW_LEN row per measurement)."""
    rows = np.asarray(rows16, dtype=np.float64)
    if tail:
        rows = rows[-tail:]
    n = float(rows[0, _lib.ROW_NSITES])
    e = rows[:, _lib.ROW_ENERGY] / n
    eta = rows[:, _lib.ROW_SUM_S] / n
    S = np.array([nematic_S(r[_lib.ROW_QXX:_lib.ROW_QXX + 6], n) for r in rows])
    return {
        "n_meas": len(rows), "energy": float(e.mean()), "eta": float(eta.mean()),
        "abs_eta": float(np.abs(eta).mean()), "S": float(S.mean()),
        "C_v": specific_heat(e, kT, n) if kT > 0 else math.nan,
        "C_v_reference": specific_heat_reference(rows[:, _lib.ROW_ETOT], kT) if kT > 0 else math.nan,
        "chi_c": chiral_susceptibility(eta, kT, n) if kT > 0 else math.nan,
    }


def summarize_batch(moments, specs) -> list[dict]:
    """Observables per replica from chll_batch_moments rows."""
    out = []
    for row, sp in zip(np.asarray(moments), specs):
        n = float(sp["ni"] * sp["nj"] * sp["nk"])
        m = row[B_NMEAS]
        kT = float(sp["kT"])
        if m > 0:
            e, e2 = row[B_SUM_E] / m, row[B_SUM_E2] / m
            eta, eta2 = row[B_SUM_ETA] / m, row[B_SUM_ETA2] / m
            S, S2 = row[B_SUM_S] / m, row[B_SUM_S2] / m
            cv = n * (e2 - e * e) / (kT * kT) if kT > 0 else math.nan
            chi = n * (eta2 - eta * eta) / kT if kT > 0 else math.nan
        else:
            e = eta = S = cv = chi = math.nan
        out.append({"kT": kT, "g": float(sp["g"]), "K": float(sp["K"]), "shape":
                    (sp["ni"], sp["nj"], sp["nk"]), "n_meas": int(m), "energy": e, "eta": eta,
                    "abs_eta": row[B_SUM_ABS_ETA] / m if m > 0 else math.nan, "S": S,
                    "C_v": cv, "chi_c": chi, "d": row[B_D], "step": int(row[B_STEP]),
                    "paccept": row[B_PACCEPT], "faccept": row[B_FACCEPT],
                    "last": (row[B_LAST_E], row[B_LAST_ETA], row[B_LAST_S])})
    return out
