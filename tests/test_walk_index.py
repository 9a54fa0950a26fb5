"""The column walk's slot arithmetic (sweep_unit.cuh walk_task), restated in
Python with its 32-bit wrapping offsets: every address a task forms stays
inside the colour arrays, and the neighbours it hands each site are the ones
the site's coordinates give (open, periodic and slab-storage boundaries).
CPU only: this is the check made before the walk runs on a GPU."""
import pytest

M = 0xffffffff
def neg(x): return (-x) & M

def slot(i, j, k, hx, nj):  # storage slot of site (i,j,k) in its colour array
    return (k * nj + j) * hx + (i >> 1)

def nbr_site(i, j, k, di, dj, dk, ni, nj, nk, pxy, pz):
    a, b, c = i + di, j + dj, k + dk
    if a < 0 or a >= ni:
        if not pxy: return None
        a %= ni
    if b < 0 or b >= nj:
        if not pxy: return None
        b %= nj
    if c < 0 or c >= nk:
        if not pz: return None
        c %= nk
    return a, b, c

def _check(ni, nj, nk, pxy, pz, C, seg, k_first=0, k_end=None, cols=None):
    assert ni % 4 == 0
    hx = ni // 2; Q = hx // 2; plane = hx * nj; per_colour = plane * nk
    k_end = nk if k_end is None else k_end
    planes = k_end - k_first
    seg = max(1, min(seg, planes)); nseg = (planes + seg - 1) // seg
    ncols = Q * nj
    bad = 0; n = 0
    tasks = range(ncols * nseg) if cols is None else [c + ncols * sg for sg in range(nseg) for c in cols]
    for t in tasks:
        sg = t // ncols; col = t - sg * ncols; j = col // Q; q = col - j * Q
        k0 = k_first + sg * seg; k1 = min(k0 + seg, k_end)
        hyp = pxy or j + 1 < nj; hym = pxy or j > 0
        oyp = hx if j + 1 < nj else neg((nj - 1) * hx)
        oym = neg(hx) if j > 0 else (nj - 1) * hx
        hx0 = pxy or q > 0; hx1 = pxy or q + 1 < Q
        ox0 = M if q > 0 else 2 * Q - 1
        ox1 = 2 if q + 1 < Q else neg(2 * q)
        u = ((k0 * nj + j) * hx + 2 * q) & M
        g = col + ncols * k0
        o = (C + j + k0) & 1
        X = u  # x-row pair slot, carried from step to step
        for k in range(k0, k1):
            Z = (u - plane) & M if k > 0 else ((u + (nk - 1) * plane) & M if pz else None)
            hzp = pz or k + 1 < nk
            ozp = plane if k + 1 < nk else neg((nk - 1) * plane)
            addrs = {"own": u, "yp": (u + oyp) & M if hyp else None, "ym": (u + oym) & M if hym else None,
                     "zp": (u + ozp) & M if hzp else None, "x": X, "zm": Z}
            e = ((u + ox0) & M if hx0 else None) if o == 0 else ((u + ox1) & M if hx1 else None)
            for nm, a in list(addrs.items()) + [("e", e)]:
                if a is not None and not (0 <= a < per_colour - (0 if nm == "e" else 1)):
                    raise AssertionError("OOB", nm, a, per_colour, (ni, nj, nk, k, j, q))
            # expected neighbours of the two sites
            i0 = 4 * q + o; i1 = i0 + 2
            assert g == q + Q * (j + nj * k) and u == slot(i0, j, k, hx, nj) == 2 * g
            for w, i in enumerate((i0, i1)):
                got = {}
                # pairs: +y, -y, +z, -z, x-row pair, e
                pair = lambda a: None if a is None else (a + w)
                got[(0, 1, 0)] = pair(addrs["yp"]); got[(0, -1, 0)] = pair(addrs["ym"])
                got[(0, 0, 1)] = pair(addrs["zp"]); got[(0, 0, -1)] = pair(addrs["zm"])
                xa, xb = X, X + 1
                if o == 0:
                    got[(1, 0, 0)] = xa if w == 0 else xb; got[(-1, 0, 0)] = e if w == 0 else xa
                else:
                    got[(1, 0, 0)] = xb if w == 0 else e; got[(-1, 0, 0)] = xa if w == 0 else xb
                for d, a in got.items():
                    s = nbr_site(i, j, k, *d, ni, nj, nk, pxy, pz)
                    want = None if s is None else slot(*s, hx, nj)
                    if want != a:
                        raise AssertionError("MISMATCH", (ni, nj, nk, pxy, pz, C, seg), (i, j, k), d, a, want)
                n += 1
            X = addrs["zp"]
            u = (u + plane) & M; g += ncols; o ^= 1
    return True



SHAPES = [(4, 2, 2), (8, 8, 8), (16, 12, 8), (32, 24, 16), (20, 14, 10), (24, 16, 6), (12, 6, 4)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("pxy,pz", [(False, False), (True, True), (True, False)])
def test_walk_slots_match_site_neighbours(shape, pxy, pz):
    ni, nj, nk = shape
    if (pxy or pz) and (nj % 2 or nk % 2):
        pytest.skip("periodic lattices have even dims")
    for C in (0, 1):
        for seg in (1, 2, 3, 5, 8, 100):
            assert _check(ni, nj, nk, pxy, pz, C, seg)


def test_walk_slots_on_slab_storage():
    # planes [2, nkl+2) of nkl+3 walked, x/y periodic, z from the stored halos
    for nkl in (2, 4, 6):
        for C in (0, 1):
            for seg in (1, 3, 8):
                assert _check(16, 12, nkl + 3, True, False, C, seg, k_first=2, k_end=nkl + 2)


def test_walk_slots_on_the_480_cube_edges():
    Q, nj = 120, 480
    cols = sorted({0, 1, Q - 1, Q, 2 * Q - 1, 5 * Q + 7} | {q + Q * (nj - 1) for q in (0, 1, Q - 1)})
    for C in (0, 1):
        assert _check(480, 480, 480, True, True, C, 16, cols=cols)
