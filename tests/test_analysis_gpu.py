"""GPU analysis kernels against the reference's own analysis outputs (golden)
and the numpy oracle: shell correlations and the chirality structure factor."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "analysis_golden.npz")


def _lattice_from(nx, ny, nz, s, boundary="open"):
    from chllmodel_b200.lattice import Lattice

    ni, nj, nk = nx.shape
    lat = Lattice(ni, nj, nk, boundary=boundary)
    f4 = np.stack([nx, ny, nz, s.astype(np.float64)], axis=-1).astype(np.float32)
    lat.upload_f4(f4.transpose(2, 1, 0, 3).reshape(-1, 4))  # natural order, i fastest
    return lat


@pytest.mark.parametrize("case", [0, 1])
def test_shell_corr_matches_reference(case):
    from chllmodel_b200.analysis import shell_correlations

    g = np.load(GOLDEN)
    p = f"c{case}_"
    lat = _lattice_from(g[p + "nx"], g[p + "ny"], g[p + "nz"], g[p + "s"])
    gn, gs, c = shell_correlations(lat, int(g[p + "nshells"]))
    lat.close()
    np.testing.assert_array_equal(c, g[p + "cn"])
    # FP32 dot products, FP64 sums
    np.testing.assert_allclose(gn, g[p + "gn"], rtol=2e-6, atol=0)
    np.testing.assert_allclose(gs, g[p + "gs"], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("case", [0, 1])
def test_structure_factor_matches_reference(case):
    from chllmodel_b200.analysis import structure_factor

    g = np.load(GOLDEN)
    p = f"c{case}_"
    lat = _lattice_from(g[p + "nx"], g[p + "ny"], g[p + "nz"], g[p + "s"])
    for q, plane in enumerate(g["planes"]):
        sf, kvs = structure_factor(lat, 16, 0.0, 0.5, plane)
        np.testing.assert_allclose(kvs, g[p + "kvs"])
        np.testing.assert_allclose(sf, g[p + f"sf{q}"], rtol=1e-9, atol=1e-15)
    lat.close()


@pytest.mark.parametrize("shape,nshells,wrap", [((20, 16, 12), 5, False), ((16, 12, 10), 4, True),
                                                ((9, 5, 3), 7, False), ((8, 6, 4), 6, True)])
def test_shell_corr_matches_oracle(shape, nshells, wrap):
    """Random swept states, open and periodic images, shells beyond the lattice."""
    from chllmodel_b200.analysis import shell_correlations
    from chllmodel_b200.lattice import Lattice, coupling
    from oracle import analysis as oa

    lat = Lattice(*shape, boundary="periodic" if wrap else "open")
    lat.init_random(7)
    lat.sweep(coupling(0.4, 1.0, 0.3), 3, seed=2)
    st = lat.download_f4().astype(np.float64).reshape(shape[2], shape[1], shape[0], 4)
    st = st.transpose(2, 1, 0, 3)
    gn, gs, c = shell_correlations(lat, nshells, wrap=wrap)
    lat.close()
    rn, rs, rc = oa.shell_corr(st[..., 0], st[..., 1], st[..., 2], st[..., 3], nshells, wrap=wrap)
    np.testing.assert_array_equal(c, rc)
    ok = rc > 0
    np.testing.assert_allclose(gn[ok], rn[ok], rtol=2e-6)
    np.testing.assert_allclose(gs[ok], rs[ok], rtol=1e-11, atol=1e-13)
    assert np.all(np.isnan(gn[~ok]))


def test_analysis_rejects_bad_arguments():
    from chllmodel_b200 import _lib
    from chllmodel_b200.analysis import projection, shell_correlations
    from chllmodel_b200.lattice import Lattice

    lat = Lattice(8, 8, 8)
    with pytest.raises(_lib.ChllError, match="nshells"):
        shell_correlations(lat, 0)
    with pytest.raises(_lib.ChllError, match="nshells"):
        shell_correlations(lat, 65)
    with pytest.raises(_lib.ChllError, match="bins"):
        projection(lat, [2000, 0, 0])
    lat.close()
