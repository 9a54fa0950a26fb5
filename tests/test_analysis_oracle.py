"""The analysis oracle (oracle/analysis.py) against the reference's own
calc_n_corr / calc_s_corr / structure_factor outputs (tests/golden/
analysis_golden.npz, made by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from oracle import analysis as oa

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "analysis_golden.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("case", [0, 1])
def test_shell_corr_matches_reference(golden, case):
    g = {k[len(f"c{case}_"):]: golden[k] for k in golden.files if k.startswith(f"c{case}_")}
    gn, gs, c = oa.shell_corr(g["nx"], g["ny"], g["nz"], g["s"], int(g["nshells"]))
    np.testing.assert_allclose(c, g["cn"], rtol=0, atol=0)
    np.testing.assert_allclose(c, g["cs"], rtol=0, atol=0)
    np.testing.assert_allclose(gn, g["gn"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(gs, g["gs"], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("case", [0, 1])
def test_structure_factor_matches_reference(golden, case):
    s = golden[f"c{case}_s"]
    for q, p in enumerate(golden["planes"]):
        sf, kvs = oa.structure_factor(s, 16, 0.0, 0.5, p)
        np.testing.assert_allclose(kvs, golden[f"c{case}_kvs"], rtol=0, atol=0)
        np.testing.assert_allclose(sf, golden[f"c{case}_sf{q}"], rtol=1e-9, atol=1e-15)


def test_projection_transform_equals_direct_sum():
    """The device's method (exact integer histogram along p, then a 1-D
    transform) equals the direct sum for integer directions."""
    rng = np.random.default_rng(5)
    s = np.where(rng.random((9, 7, 6)) < 0.5, -1, 1)
    i, j, k = np.meshgrid(np.arange(1, 10), np.arange(1, 8), np.arange(1, 7), indexing="ij")
    for p in ([1, 0, 0], [1, 1, 1], [2, -1, 3], [0, -1, 1]):
        m = p[0] * i + p[1] * j + p[2] * k
        mm = np.arange(m.min(), m.max() + 1)
        hist = np.array([s[m == v].sum() for v in mm])
        kvs = np.linspace(0.0, 0.7, 11)
        sc = np.array([np.sum(hist * np.exp(-1j * kv * mm)) for kv in kvs]) / s.size
        ref, _ = oa.structure_factor(s, 11, 0.0, 0.7, p)
        np.testing.assert_allclose(sc.real ** 2 + sc.imag ** 2, ref, rtol=1e-9, atol=1e-15)


def test_periodic_shell_counts():
    rng = np.random.default_rng(2)
    shape = (6, 4, 4)
    n = rng.normal(size=(3,) + shape)
    n /= np.linalg.norm(n, axis=0)
    s = np.where(rng.random(shape) < 0.5, -1, 1)
    gn, gs, c = oa.shell_corr(n[0], n[1], n[2], s, 3, wrap=True)
    r2 = [di * di + dj * dj + dk * dk for di in range(-2, 3) for dj in range(-2, 3)
          for dk in range(-2, 3)]
    expect = np.bincount([int(np.floor(np.sqrt(v))) for v in r2 if v < 9], minlength=3)
    np.testing.assert_array_equal(c, expect * s.size)
    assert gn[0] == pytest.approx(1.0, rel=1e-14)
