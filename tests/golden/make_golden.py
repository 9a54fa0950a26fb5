"""Generates the committed golden fixtures under tests/golden/.

Run with the path of a mdeutsc2/ChLLModel checkout
(``python tests/golden/make_golden.py --reference PATH``, or the
environment variable CHLL_REFERENCE_TREE); the fixtures it writes are small
and committed, and nothing at test time reads the reference tree.

1. ``ekernel_energy.npz`` -- the reference's own independent restatement of
   the local site energy, the numba stencil ``ekernel`` in
   notebooks/paper_plots2.ipynb (cell 0), executed here on seeded random
   lattices.  The cell's source is read from the notebook and its stencil is
   evaluated site by site with relative indexing (numba is not installed; the
   arithmetic is the notebook's own Python code).  Expected values are given
   for interior sites, where the stencil and chll_mod.f90:363-412 agree
   (the stencil fixes KK = 1.0 and has no field term).
2. ``philox_kat.json`` -- the published Philox4x32-10 known-answer vectors
   (Salmon et al., SC'11, Random123 distribution).
4. ``chi_golden.npz`` -- the reference's own measure_chi
   (notebooks/.ipynb_checkpoints/Xch-checkpoint.ipynb, cell 2: chiral
   susceptibility, mean enantiomeric excess and specific heat from the macro
   CSV files) run on seeded CSV files in ChLLSim's format, its matplotlib
   calls recorded instead of drawn.
3. ``analysis_golden.npz`` -- the reference's own analysis functions run on
   small seeded fields: calc_n_corr / calc_s_corr (notebooks/paper_plots2.ipynb,
   cell 0) and structure_factor / get_sc
   (notebooks/.ipynb_checkpoints/hero_stripe-checkpoint.py).  Their source is
   read from those files and executed with the numba decorators and tqdm
   replaced by identities (plain Python on the same arithmetic).  Directors
   are FP32 values stored as FP64, so the FP32 device state holds them exactly.
"""
from __future__ import annotations

import json
import os
import re
import textwrap

import numpy as np

REF = os.environ.get("CHLL_REFERENCE_TREE", "")  # set by main() from --reference
HERE = os.path.dirname(os.path.abspath(__file__))


def _ekernel_source() -> str:
    nb = json.load(open(os.path.join(REF, "notebooks", "paper_plots2.ipynb")))
    src = "".join(nb["cells"][0]["source"])
    m = re.search(r"@stencil\s*\ndef ekernel\(.*?\n(?=\S)", src + "\nEND", re.S)
    if not m:
        raise RuntimeError("ekernel not found in paper_plots2.ipynb cell 0")
    body = m.group(0).replace("@stencil\n", "")
    return textwrap.dedent(body)


class _Rel:
    """Relative-index view of an array around one centre site."""

    def __init__(self, a, i, j, k):
        self.a, self.i, self.j, self.k = a, i, j, k

    def __getitem__(self, idx):
        di, dj, dk = idx
        return self.a[self.i + di, self.j + dj, self.k + dk]


def make_ekernel_fixture(path):
    ns: dict = {}
    exec(_ekernel_source(), ns)  # the reference notebook's ekernel function
    ekernel = ns["ekernel"]
    cases = []
    rng = np.random.default_rng(20240611)
    for shape in [(5, 5, 5), (6, 4, 5), (7, 6, 4)]:
        ni, nj, nk = shape
        ct = rng.uniform(-1, 1, shape)
        st = np.sqrt(1 - ct * ct)
        ph = rng.uniform(0, 2 * np.pi, shape)
        nx, ny, nz = st * np.cos(ph), st * np.sin(ph), ct
        s = np.where(rng.random(shape) < 0.5, -1, 1).astype(np.int32)
        e = np.full(shape, np.nan)
        for i in range(1, ni - 1):
            for j in range(1, nj - 1):
                for k in range(1, nk - 1):
                    e[i, j, k] = ekernel(_Rel(nx, i, j, k), _Rel(ny, i, j, k),
                                         _Rel(nz, i, j, k), _Rel(s, i, j, k))
        cases.append(dict(nx=nx, ny=ny, nz=nz, s=s, e=e))
    out = {}
    for c, d in enumerate(cases):
        for key, val in d.items():
            out[f"c{c}_{key}"] = val
    out["ncases"] = np.int64(len(cases))
    out["KK"] = np.float64(1.0)
    np.savez_compressed(path, **out)


PHILOX_KAT = [
    # counter (4 words), key (2 words), output (4 words)
    [[0x00000000, 0x00000000, 0x00000000, 0x00000000], [0x00000000, 0x00000000],
     [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]],
    [[0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF], [0xFFFFFFFF, 0xFFFFFFFF],
     [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]],
    [[0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]],
]


def _def_source(src: str, name: str) -> str:
    """Source of top-level function `name` (without decorators) in `src`."""
    lines = src.split("\n")
    start = next(i for i, l in enumerate(lines) if l.startswith(f"def {name}("))
    end = start + 1
    while end < len(lines) and (not lines[end].strip() or lines[end][0] in " \t"):
        end += 1
    return "\n".join(lines[start:end]) + "\n"


def _identity_decorator(*args, **kwargs):
    if len(args) == 1 and callable(args[0]) and not kwargs:
        return args[0]
    return lambda f: f


def _reference_analysis():
    nb = json.load(open(os.path.join(REF, "notebooks", "paper_plots2.ipynb")))
    cell = "".join(nb["cells"][0]["source"])
    hero = open(os.path.join(REF, "notebooks", ".ipynb_checkpoints",
                             "hero_stripe-checkpoint.py")).read()
    ns = {"np": np, "jit": _identity_decorator, "njit": _identity_decorator, "prange": range,
          "tqdm": lambda x: x}
    for name in ("calc_n_corr", "calc_s_corr"):
        exec(_def_source(cell, name), ns)
    for name in ("get_sc", "structure_factor"):
        exec(_def_source(hero, name), ns)
    return ns


def make_analysis_fixture(path):
    ns = _reference_analysis()
    rng = np.random.default_rng(20251203)
    out = {}
    cases = [((6, 5, 4), 3), ((7, 6, 5), 4)]
    planes = [[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1], [1, -1, 1], [1, 1, -1]]
    for c, (shape, nshells) in enumerate(cases):
        ct_ = rng.uniform(-1, 1, shape).astype(np.float32)
        st = np.sqrt(np.float32(1) - ct_ * ct_)
        ph = rng.uniform(0, 2 * np.pi, shape).astype(np.float32)
        nx = (st * np.cos(ph)).astype(np.float32).astype(np.float64)
        ny = (st * np.sin(ph)).astype(np.float32).astype(np.float64)
        nz = ct_.astype(np.float64)
        s = np.where(rng.random(shape) < 0.45, -1, 1).astype(np.int32)
        gn, cn = ns["calc_n_corr"](nx, ny, nz, nshells)
        gs, cs = ns["calc_s_corr"](s, nshells)
        out.update({f"c{c}_nx": nx, f"c{c}_ny": ny, f"c{c}_nz": nz, f"c{c}_s": s,
                    f"c{c}_nshells": np.int64(nshells), f"c{c}_gn": gn, f"c{c}_cn": cn,
                    f"c{c}_gs": gs, f"c{c}_cs": cs})
        for q, p in enumerate(planes):
            sf, kvs = ns["structure_factor"](s, 16, 0.0, 0.5, p)
            out[f"c{c}_sf{q}"] = sf
        out[f"c{c}_kvs"] = kvs
    out["ncases"] = np.int64(len(cases))
    out["planes"] = np.asarray(planes, np.int64)
    np.savez_compressed(path, **out)


class _Recorder:
    """Stands in for matplotlib: every call returns itself, and the scatter()
    calls' arguments are kept (measure_chi plots its results)."""

    def __init__(self):
        self.scatters = []

    def subplots(self, *a, **k):
        return self, (self, self, self)

    def scatter(self, x, y, *a, **k):
        self.scatters.append((list(x), list(y)))

    def __getattr__(self, name):
        return lambda *a, **k: self


def make_chi_fixture(path):
    """The reference's measure_chi (notebooks/.ipynb_checkpoints/
    Xch-checkpoint.ipynb, cell 2: chiral susceptibility, mean excess and
    specific heat from the macro CSVs) run on seeded CSVs written in
    ChLLSim's format (Step,TotalEnergy,Eexcess,Paccept,Faccept,D), with
    load_csv from cell 0."""
    import tempfile

    nb = json.load(open(os.path.join(REF, "notebooks", ".ipynb_checkpoints",
                                     "Xch-checkpoint.ipynb")))
    cell0 = "".join(nb["cells"][0]["source"])
    cell2 = "".join(nb["cells"][2]["source"])
    load_src = cell0[cell0.index("def load_csv"):cell0.index("def plot_energy")]
    chi_src = cell2[cell2.index("def measure_chi"):cell2.index("measure_chi(0.001)")]
    rng = np.random.default_rng(20251204)
    points = [(1.0, 0.3), (1.0, 0.7), (1.0, 1.3), (0.1, 0.5)]
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "nb"))
        files = []
        for q, (K, kbt) in enumerate(points):
            name = f"aligned_K{K}_kbt{kbt}"
            os.makedirs(os.path.join(tmp, "data", name))
            rows = np.column_stack([
                np.arange(1, 201) * 50,
                rng.normal(-1.5, 0.02, 200),        # TotalEnergy (per site)
                rng.normal(0.1 * q, 0.05, 200),     # Eexcess
                rng.uniform(0.3, 0.7, 200), rng.uniform(0.3, 0.7, 200),
                rng.uniform(0.05, 0.2, 200)])
            rel = f"../data/{name}/{name}.csv"
            with open(os.path.join(tmp, "data", name, f"{name}.csv"), "w") as f:
                f.write("Step,TotalEnergy,Eexcess,Paccept,Faccept,D\n")
                for r in rows:
                    f.write(f"{int(r[0])}," + ",".join(repr(float(v)) for v in r[1:]) + "\n")
            files.append(rel)
            out[f"p{q}_rows"] = rows
        cwd = os.getcwd()
        os.chdir(os.path.join(tmp, "nb"))
        try:
            rec = _Recorder()
            ns = {"np": np, "plt": rec, "csvfiles": sorted(files)}
            exec(load_src + chi_src, ns)
            for K in sorted({p[0] for p in points}):
                rec.scatters = []
                ns["measure_chi"](K)
                (kbts, chi), (_, ent), (_, cv) = rec.scatters
                out[f"K{K}_kbts"] = np.asarray(kbts)
                out[f"K{K}_chi"] = np.asarray(chi)
                out[f"K{K}_excess"] = np.asarray(ent)
                out[f"K{K}_cv"] = np.asarray(cv)
        finally:
            os.chdir(cwd)
    out["points"] = np.asarray(points)
    np.savez_compressed(path, **out)


def main():
    global REF
    import argparse

    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=REF,
                    help="path of a mdeutsc2/ChLLModel checkout (or CHLL_REFERENCE_TREE)")
    REF = ap.parse_args().reference
    if not REF or not os.path.isdir(os.path.join(REF, "notebooks")):
        ap.error("give --reference PATH (or CHLL_REFERENCE_TREE): a ChLLModel checkout")
    make_ekernel_fixture(os.path.join(HERE, "ekernel_energy.npz"))
    make_analysis_fixture(os.path.join(HERE, "analysis_golden.npz"))
    make_chi_fixture(os.path.join(HERE, "chi_golden.npz"))
    with open(os.path.join(HERE, "philox_kat.json"), "w") as f:
        json.dump({"generator": "philox4x32-10", "vectors": PHILOX_KAT}, f, indent=1)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
