"""CPU tests of the C ABI: the library loads, exports every symbol the
header declares, validates arguments before touching a device, fails loudly
without a GPU, and its host-only reference entry point ``init`` builds the
same sublattice lists as chll_mod.f90:9-38."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu


def header_functions():
    src = open(os.path.join(ROOT, "include", "chll_mod.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", src)
    return sorted(set(n for n in names if n not in ("if", "while", "sizeof")))


def test_library_exports_every_declared_symbol():
    from chllmodel_b200 import _lib

    L = _lib.load()
    declared = header_functions()
    assert "init" in declared and "run" in declared
    for name in declared:
        assert hasattr(L, name), f"libchll_mod.so does not export {name}"
    assert sorted(_lib.EXPORTS) == declared


def test_version_and_status():
    from chllmodel_b200 import _lib

    L = _lib.load()
    assert b"sm_100a" in L.chll_version()
    assert L.chll_last_status() in range(6)


def test_init_sublattices_match_reference_rule():
    from chllmodel_b200 import chll

    for (ni, nj, nk) in [(4, 4, 4), (5, 3, 2), (6, 5, 7)]:
        n = ni * nj * nk
        sim = chll.ChLLSim(ni, nj, nk, 0.5, 0.1, 0.5, 0.0, 0.0, verbose=False)
        sim.init_with_s(np.ones((ni, nj, nk), np.int32))
        i, j, k = np.meshgrid(np.arange(1, ni + 1), np.arange(1, nj + 1), np.arange(1, nk + 1),
                              indexing="ij")
        idx = (i + (j - 1) * ni + (k - 1) * ni * nj).ravel(order="F")
        odd = ((i + j + k) % 2 != 0).ravel(order="F")
        n1 = int(odd.sum())
        assert np.array_equal(sim.sl1[:n1], idx[odd][: sim.nsub])
        if n % 2 == 0:
            assert np.array_equal(sim.sl2, idx[~odd])
        # directors default to x-hat when never initialised (chll/chll.py:91-98)
        assert np.all(sim.nx == 1.0) and np.all(sim.ny == 0.0)


def test_argument_validation_without_device():
    from chllmodel_b200 import _lib

    L = _lib.load()
    h = ct.c_void_p()
    rc = L.chll_lattice_create(7, 8, 8, _lib.CHLL_PERIODIC, ct.byref(h))
    assert rc == _lib.CHLL_EINVAL and b"even" in L.chll_last_error()
    rc = L.chll_lattice_create(0, 8, 8, _lib.CHLL_OPEN, ct.byref(h))
    assert rc == _lib.CHLL_EINVAL
    rc = L.chll_lattice_create(8, 8, 8, 7, ct.byref(h))
    assert rc == _lib.CHLL_EINVAL
    # 32-bit slot indices: 1 x 46341 x 46341 has < 2^32 sites, but its rows
    # pad to 4 sites, 2^31+ slots per colour
    rc = L.chll_lattice_create(1, 46341, 46341, _lib.CHLL_OPEN, ct.byref(h))
    assert rc == _lib.CHLL_EINVAL and b"slots per colour" in L.chll_last_error()
    # the whole 4 x 16384 x 65534 lattice fits; as one slab its 3 halo planes do not
    rc = L.chll_lattice_create_slab(4, 16384, 65534, 0, 65534, _lib.CHLL_OPEN, ct.byref(h))
    assert rc == _lib.CHLL_EINVAL and b"halo planes" in L.chll_last_error()
    # a batch replica of 2^30 units (2^31 slots per colour) is refused before any device call
    spec = (_lib.ReplicaSpec * 1)(_lib.ReplicaSpec(4096, 4096, 256, _lib.CHLL_PERIODIC, 1.0, 1.0,
                                                   0.0, 1.0, 0.1, 1, 0, 0))
    rc = L.chll_batch_create(spec, 1, ct.byref(h))
    assert rc == _lib.CHLL_EINVAL and b"limit 2^30" in L.chll_last_error()
    cfg = _lib.RunConfig(0.5, 0.5, 0.0, 1.0, 0.1, 1, 0, 0, 10000, 0, 0)
    z = np.zeros((4, 4, 4), order="F")
    p = z.ctypes.data_as(ct.c_void_p)
    rc = L.chll_run_ex(ct.byref(cfg), 1, 10, 0, p, p, p, p, 4, 4, 4, None, None, None, None)
    assert rc == _lib.CHLL_EINVAL and b"nout" in L.chll_last_error()


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure path")
def test_fails_loudly_without_gpu(capfd):
    from chllmodel_b200 import _lib, chll
    from chllmodel_b200.lattice import Lattice

    with pytest.raises(_lib.ChllError, match="no CUDA device"):
        Lattice(8, 8, 8)
    sim = chll.ChLLSim(4, 4, 4, 0.5, 0.1, 0.5, 0.0, 0.0, verbose=False)
    sim.init_rand_s()
    with pytest.raises(_lib.ChllError, match="no CUDA device"):
        sim.run(10, 5)
    # the reference entry point itself reports on stderr and returns
    d = ct.c_double(0.1)
    msteps = np.zeros(2, np.int32)
    m = np.zeros((2, 5), order="F")
    chll.ftn_run(ct.c_int(1), ct.c_int(10), ct.c_int(5), sim.nx, sim.ny, sim.nz, sim.s,
                 sim.dope, sim.sl1, sim.sl2, ct.c_double(0.0), ct.c_double(0.5), d,
                 ct.c_double(0.5), ct.c_int(4), ct.c_int(4), ct.c_int(4), ct.c_int(32),
                 msteps, m)
    assert chll.libchll_mod.chll_last_status() == _lib.CHLL_ECUDA
    assert "no CUDA device" in capfd.readouterr().err


def test_chllsim_files(tmp_path):
    from chllmodel_b200 import chll

    data = tmp_path / "data"
    data.mkdir()
    sim = chll.ChLLSim(4, 4, 4, 0.5, 0.1, 0.5, 0.25, 0.0, name="t1", data_folder=str(data),
                       verbose=False)
    sim.save_params(100, 10)
    txt = (data / "t1" / "t1t1_params.txt").read_text().splitlines()
    assert txt[0] == "t1" and txt[1] == "nsteps = 100 nout = 10"
    assert txt[2] == "ni,nj,nk = 4 4 4" and txt[6] == "g = 0.25"
    sim.msteps = np.array([10, 20], np.int32)
    sim.m = np.asfortranarray(np.arange(10, dtype=np.float64).reshape(2, 5))
    sim.save_macros()
    lines = (data / "t1" / "t1.csv").read_text().splitlines()
    assert lines[0] == "Step,TotalEnergy,Eexcess,Paccept,Faccept,D"
    assert lines[1] == "10,0.0,1.0,2.0,3.0,4.0"
    sim.nx[:] = 0.5
    sim.save_config()
    sim2 = chll.ChLLSim(4, 4, 4, 0.5, 0.1, 0.5, 0.25, 0.0, name="t2", data_folder=str(data),
                        verbose=False)
    s = sim2.load_config(str(data / "t1" / "t1_data.npz"))
    assert np.all(sim2.nx == 0.5) and s.dtype == np.int32
    with pytest.raises(chll.ChllError):
        chll.ChLLSim(4, 4, 4, 0.5, 0.1, 0.5, 0.25, 0.0, name="t1", data_folder=str(data),
                     verbose=False)
