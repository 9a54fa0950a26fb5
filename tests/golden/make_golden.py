"""Generates the committed golden fixtures under tests/golden/.

Run in a checkout that has the reference tree at /root/reference
(``python tests/golden/make_golden.py``); the fixtures it writes are small
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
"""
from __future__ import annotations

import json
import os
import re
import textwrap

import numpy as np

REF = "/root/reference"
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


def main():
    make_ekernel_fixture(os.path.join(HERE, "ekernel_energy.npz"))
    with open(os.path.join(HERE, "philox_kat.json"), "w") as f:
        json.dump({"generator": "philox4x32-10", "vectors": PHILOX_KAT}, f, indent=1)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
