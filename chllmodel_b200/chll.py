"""``ChLLSim``: the reference's Python host class over the B200 library.

Mirrors ``class ChLLSim`` of the reference (chll/chll.py:38-306) -- same
constructor, attributes, methods, ctypes prototypes ``ftn_init``/``ftn_run``
(chll/chll.py:9-36) and NPZ/CSV/params files -- with libchll_mod.so built
for sm_100a underneath.  Scripts written against the reference run
unchanged (``from chllmodel_b200 import chll; chll.ChLLSim(...)``).

Differences, all additive:
  * keyword-only options ``seed``, ``boundary`` ('open' as the reference
    sweep, or 'periodic'), ``epsilon``, ``adapt_until`` and ``verbose``;
    with the defaults ``run`` goes through the reference's own ``run``
    entry point;
  * ``run`` works with ``name=None`` (the reference crashes in
    ``save_params``, chll/chll.py:141,155) and writes the adapted step size
    back to ``self.d``, plus the seed/step/d needed for an exact resume
    into the NPZ (``save_config``) next to the reference's keys;
  * ``init()`` is accepted as an alias of ``init_rand_s()`` (several
    reference drivers call it, e.g. scripts/phase_diagram.py:29);
  * ``self.rows`` holds the FP64 observables row of every measurement
    (energy, sum of s, Q-tensor moments) for ``observables.summarize``.
Errors are raised as ``ChllError`` instead of calling ``exit()``.
"""
from __future__ import annotations

import ctypes as ct
import os
import time

import numpy as np
from numpy import ctypeslib

from . import _lib
from ._lib import ChllError, RunConfig, check

# the shared library and its two reference entry points
libchll_mod = _lib.load()

ftn_init = libchll_mod.init
ftn_init.argtypes = [ctypeslib.ndpointer(dtype=np.float64, ndim=3, flags="F_CONTIGUOUS"),  # nx
                     ctypeslib.ndpointer(dtype=np.float64, ndim=3, flags="F_CONTIGUOUS"),  # ny
                     ctypeslib.ndpointer(dtype=np.float64, ndim=3, flags="F_CONTIGUOUS"),  # nz
                     ctypeslib.ndpointer(dtype=np.int32, ndim=3, flags="F_CONTIGUOUS"),    # s
                     ctypeslib.ndpointer(dtype=np.int32, ndim=3, flags="F_CONTIGUOUS"),    # dope
                     ctypeslib.ndpointer(dtype=np.int32, ndim=1, flags="F_CONTIGUOUS"),    # sl1
                     ctypeslib.ndpointer(dtype=np.int32, ndim=1, flags="F_CONTIGUOUS"),    # sl2
                     ct.POINTER(ct.c_int), ct.POINTER(ct.c_int), ct.POINTER(ct.c_int),
                     ct.POINTER(ct.c_int)]
ftn_init.restype = None

ftn_run = libchll_mod.run
ftn_run.argtypes = [ct.POINTER(ct.c_int), ct.POINTER(ct.c_int), ct.POINTER(ct.c_int),  # nstart,nstop,nout
                    ctypeslib.ndpointer(dtype=np.float64, ndim=3, flags="F_CONTIGUOUS"),  # nx
                    ctypeslib.ndpointer(dtype=np.float64, ndim=3, flags="F_CONTIGUOUS"),  # ny
                    ctypeslib.ndpointer(dtype=np.float64, ndim=3, flags="F_CONTIGUOUS"),  # nz
                    ctypeslib.ndpointer(dtype=np.int32, ndim=3, flags="F_CONTIGUOUS"),    # s
                    ctypeslib.ndpointer(dtype=np.int32, ndim=3, flags="F_CONTIGUOUS"),    # dope
                    ctypeslib.ndpointer(dtype=np.int32, ndim=1, flags="F_CONTIGUOUS"),    # sl1
                    ctypeslib.ndpointer(dtype=np.int32, ndim=1, flags="F_CONTIGUOUS"),    # sl2
                    ct.POINTER(ct.c_double),  # g
                    ct.POINTER(ct.c_double),  # KK
                    ct.POINTER(ct.c_double),  # d
                    ct.POINTER(ct.c_double),  # kbt
                    ct.POINTER(ct.c_int), ct.POINTER(ct.c_int), ct.POINTER(ct.c_int),
                    ct.POINTER(ct.c_int),
                    ctypeslib.ndpointer(dtype=np.int32, ndim=1, flags="F_CONTIGUOUS"),
                    ctypeslib.ndpointer(dtype=np.float64, ndim=2, flags="F_CONTIGUOUS")]
ftn_run.restype = None


def set_seed(seed: int) -> None:
    """Seed of the Philox stream used by the reference-style ``run``."""
    libchll_mod.chll_set_seed(int(seed))


class ChLLSim:
    def __init__(self, ni, nj, nk, kbt, d, KK, g, rho, name=None, overwrite=False, *,
                 seed=None, boundary="open", epsilon=1.0, adapt_until=10000, verbose=True,
                 data_folder="./data"):
        # parameters (chll/chll.py:40-49)
        self.name = name
        self.ni = ni
        self.nj = nj
        self.nk = nk
        self.kbt = kbt
        self.d = d
        self.KK = KK
        self.g = g
        self.rho = rho
        # extensions
        if boundary not in ("open", "periodic"):
            raise ValueError("boundary must be 'open' or 'periodic'")
        self.seed = seed
        self.boundary = boundary
        self.epsilon = float(epsilon)
        self.adapt_until = int(adapt_until)
        self.verbose = verbose
        self.data_folder = data_folder
        self.step = 0

        # internal parameters
        self.overwrite = overwrite
        self.simpath = None
        self.nsub = int((self.ni * self.nj * self.nk) / 2)

        # arrays, F-contiguous as the Fortran side expects (chll/chll.py:57-82)
        shape = (self.ni, self.nj, self.nk)
        self.nx = np.zeros(shape, dtype=np.float64, order="F")
        self.ny = np.zeros(shape, dtype=np.float64, order="F")
        self.nz = np.zeros(shape, dtype=np.float64, order="F")
        self.s = np.zeros(shape, dtype=np.int32, order="F")
        self.dope = np.zeros(shape, dtype=np.int32, order="F")
        self.sl1 = np.zeros(self.nsub, dtype=np.int32, order="F")
        self.sl2 = np.zeros(self.nsub, dtype=np.int32, order="F")

        self.m = None  # measurables
        self.msteps = None
        self.rows = None
        self.setup_folders()

    def _log(self, msg):
        if self.verbose:
            print(msg)

    # -- initial state (chll/chll.py:84-115) ------------------------------
    def _default_directors(self):
        if np.mean(np.sqrt(self.nx * self.nx + self.ny * self.ny + self.nz * self.nz)) == 0.0:
            self._log("> Nx,Ny,Nz not initialized, setting nx[:,:,:] = 1.0")
            self.nx[:, :, :] = 1.0
            self.ny[:, :, :] = 0.0
            self.nz[:, :, :] = 0.0

    def _ftn_init(self):
        ftn_init(self.nx, self.ny, self.nz, self.s, self.dope, self.sl1, self.sl2,
                 ct.c_int(self.ni), ct.c_int(self.nj), ct.c_int(self.nk), ct.c_int(self.nsub))
        check(libchll_mod.chll_last_status())

    def init_rand_s(self):
        """s = +1, or -1 with probability 1/2, per site (chll/chll.py:84-101)."""
        flip = np.random.rand(self.ni, self.nj, self.nk) < 0.5
        self.s[:, :, :] = np.where(flip, -1, 1).astype(np.int32)
        self._default_directors()
        self._ftn_init()
        self._log("> Init Done!")

    def init(self):
        """Alias of init_rand_s() for drivers that call sim.init()."""
        self.init_rand_s()

    def init_with_s(self, init_s):
        self.s[:, :, :] = init_s
        self._default_directors()
        self._ftn_init()
        self._log("> Init Done!")

    def init_random_directors(self, rng=None):
        """Directors uniform on the sphere, as the drivers' init_random
        (e.g. scripts/pdanneal.py:5-16), vectorised."""
        rng = np.random if rng is None else rng
        shape = (self.ni, self.nj, self.nk)
        costh = 2.0 * (rng.random_sample(shape) - 0.5) if rng is np.random else \
            2.0 * (rng.random(shape) - 0.5)
        sinth = np.sqrt(1.0 - costh * costh)
        phi = (rng.random_sample(shape) if rng is np.random else rng.random(shape)) * 2 * np.pi
        self.nx[:, :, :] = sinth * np.cos(phi)
        self.ny[:, :, :] = sinth * np.sin(phi)
        self.nz[:, :, :] = costh

    # -- files (chll/chll.py:117-151) ---------------------------------------
    def setup_folders(self):
        data_folder = self.data_folder
        if self.name is None:
            self._log("> Not saving sim")
            return
        if not os.path.exists(data_folder):
            raise ChllError(_lib.CHLL_EINVAL, f"'{data_folder}' does not exist.")
        simname_folder_path = os.path.join(data_folder, self.name)
        if os.path.exists(simname_folder_path):
            self._log(f"> ERROR: '{self.name}' in '{data_folder}'!")
            if not self.overwrite:
                raise ChllError(_lib.CHLL_EINVAL,
                                f"'{self.name}' exists in '{data_folder}' and overwrite=False")
            self._log(f"> Overwriting '{self.name}' in '{data_folder}' ... ")
        os.makedirs(simname_folder_path, exist_ok=True)
        self._log(f"> {simname_folder_path}")
        self.simpath = simname_folder_path

    def save_params(self, nsteps, nout):
        if self.name is None:
            return
        params_name = self.name + self.name + "_params.txt"
        with open(os.path.join(self.simpath, params_name), "w") as f:
            f.write(self.name + "\n")
            f.write("nsteps = " + str(nsteps) + " nout = " + str(nout) + "\n")
            f.write("ni,nj,nk = " + str(self.ni) + " " + str(self.nj) + " " + str(self.nk) + "\n")
            f.write("kbt = " + str(self.kbt) + "\n")
            f.write("d = " + str(self.d) + "\n")
            f.write("KK = " + str(self.KK) + "\n")
            f.write("g = " + str(self.g) + "\n")
            f.write("rho = " + str(self.rho) + "\n")

    # -- the hot path (chll/chll.py:154-178) --------------------------------
    def _reference_call(self) -> bool:
        return (self.seed is None and self.boundary == "open" and self.epsilon == 1.0
                and self.adapt_until == 10000 and self.verbose)

    def run(self, nsteps, nout, save=False, nstart=1):
        self.save_params(nsteps, nout)
        nstop = nstart + nsteps - 1
        rows = int(nsteps / nout)
        self.msteps = np.zeros(rows, dtype=np.int32, order="F")
        self.m = np.zeros((rows, 5), dtype=np.float64, order="F")
        self.rows = np.zeros((rows, _lib.ROW_LEN), dtype=np.float64)
        self._log("> RUNNING")
        st = time.perf_counter()
        if self._reference_call() and nstart == 1:
            d = ct.c_double(self.d)
            ftn_run(ct.c_int(nstart), ct.c_int(nstop), ct.c_int(nout),
                    self.nx, self.ny, self.nz, self.s, self.dope, self.sl1, self.sl2,
                    ct.c_double(self.g), ct.c_double(self.KK), d, ct.c_double(self.kbt),
                    ct.c_int(self.ni), ct.c_int(self.nj), ct.c_int(self.nk), ct.c_int(self.nsub),
                    self.msteps, self.m)
            check(libchll_mod.chll_last_status())
            self.rows = None
            self.d = d.value
        else:
            cfg = RunConfig(float(self.kbt), float(self.KK), float(self.g), float(self.epsilon),
                            float(self.d), int(self.seed if self.seed is not None else 1), 0,
                            _lib.CHLL_PERIODIC if self.boundary == "periodic" else _lib.CHLL_OPEN,
                            int(self.adapt_until), int(bool(self.verbose)), 0)
            d_out = ct.c_double()
            ptr = lambda a: a.ctypes.data_as(ct.c_void_p)
            check(libchll_mod.chll_run_ex(ct.byref(cfg), int(nstart), int(nstop), int(nout),
                                          ptr(self.nx), ptr(self.ny), ptr(self.nz), ptr(self.s),
                                          self.ni, self.nj, self.nk, ptr(self.msteps),
                                          ptr(self.m), ptr(self.rows), ct.byref(d_out)))
            self.d = d_out.value
        self.step = nstop
        et = time.perf_counter()
        if save:
            self.save_macros()
            self.save_config()
        self._log(f"> DONE!  {et - st}")
        return et - st

    # -- outputs (chll/chll.py:198-262) -------------------------------------
    def _checked_path(self, fname):
        if not os.path.exists(self.simpath):
            raise ChllError(_lib.CHLL_EINVAL, f"'{self.simpath}' does not exist")
        path = os.path.join(self.simpath, fname)
        if os.path.isfile(path) and not self.overwrite:
            raise ChllError(_lib.CHLL_EINVAL, f"'{path}' exists and overwrite=False")
        return path

    def save_config(self):
        if self.name is None:
            return
        path = self._checked_path(self.name + "_data.npz")
        np.savez_compressed(path, nx=self.nx, ny=self.ny, nz=self.nz, s=self.s, dope=self.dope,
                            seed=np.int64(self.seed if self.seed is not None else -1),
                            step=np.int64(self.step), d=np.float64(self.d))
        self._log(f"> Wrote '{path}'")

    def save_macros(self):
        if self.name is None:
            return
        path = self._checked_path(self.name + ".csv")
        with open(path, "w") as fcsv:
            fcsv.write("Step,TotalEnergy,Eexcess,Paccept,Faccept,D\n")
            for i in range(len(self.msteps)):
                fcsv.write(str(int(self.msteps[i])) + "," + str(self.m[i, 0]) + "," +
                           str(self.m[i, 1]) + "," + str(self.m[i, 2]) + "," +
                           str(self.m[i, 3]) + "," + str(self.m[i, 4]) + "\n")
        self._log(f"> Wrote '{path}'")

    def load_config(self, path):
        """Loads an NPZ written by save_config (reference keys nx,ny,nz,s,dope;
        seed/step/d when present) and returns the chirality array."""
        data = np.load(path)
        self.nx[:, :, :] = data["nx"]
        self.ny[:, :, :] = data["ny"]
        self.nz[:, :, :] = data["nz"]
        if "dope" in data:
            self.dope[:, :, :] = data["dope"]
        if "d" in data:
            self.d = float(data["d"])
        if "step" in data:
            self.step = int(data["step"])
        if "seed" in data and int(data["seed"]) >= 0:
            self.seed = int(data["seed"])
        return np.array(data["s"], dtype=np.int32)

    def plot_config(self):
        import matplotlib.pyplot as plt

        X, Z = np.meshgrid(np.arange(0, self.ni), np.arange(0, self.nk))
        mp = int(np.floor(self.nj / 2))
        u = self.nx[:, mp, :]
        w = self.nz[:, mp, :]
        s_color = self.s[:, mp, :]
        fig = plt.figure(figsize=(10, 10))
        ax = fig.add_subplot(111)
        q = ax.quiver(X, Z, u, w, s_color, pivot="mid", headlength=0, headwidth=0,
                      headaxislength=0, scale_units="xy", scale=0.75, cmap="coolwarm")
        ax.set_xlabel("X")
        ax.set_ylabel("Z")
        ax.set_title(self.name)
        fig.colorbar(q)
        if self.simpath:
            plt.savefig(os.path.join(self.simpath, self.name + ".png"))
        plt.close(fig)

    def output_old(self):
        scale = 0.4
        j = int(self.nj / 2)
        with open(self.name + "a.dat", "w") as fa, open(self.name + "b.dat", "w") as fb:
            for i in range(self.ni):
                for k in range(self.nk):
                    x1 = i - scale * self.nx[i, j, k]
                    x2 = i + scale * self.nx[i, j, k]
                    z1 = k - scale * self.nz[i, j, k]
                    z2 = k + scale * self.nz[i, j, k]
                    f = fa if self.s[i, j, k] == 1 else fb
                    f.write(f"{x1} {z1}\n{x2} {z2}\n\n")
