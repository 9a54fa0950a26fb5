"""One lattice split into z-slabs: over the GPUs of a node, or several slabs in
one process.

Each slab holds global planes z0 .. z0+nkl-1 plus a halo plane on each side
(``chll_lattice_create_slab``) and draws the random counters of its global
sites, so slabs that refresh their halos between passes follow exactly the
chain of the whole lattice swept on one GPU.  Per sweep (the fused form):

  pass A on every slab -> halo exchange of colour 0 -> sum the flip count
  over slabs -> control update;  pass B -> halo exchange of colour 1 -> sum
  the director count -> control update (paccept, d, step);

and after the last sweep the closing flip pass F, its halo exchange and count.
A halo exchange moves one plane of one colour (hx*nj float4) to each
neighbouring slab; a count sum is a 64-bit all-reduce.  ``LocalHalo`` does both
for slabs held by this process (device-to-device copies on one stream);
``TorchHalo`` does them with ``torch.distributed`` (NCCL between GPUs, or gloo
with host tensors) for one slab per rank.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib
from ._lib import check
from .lattice import FUSED_A, FUSED_A0, FUSED_B, FUSED_F, Lattice

LOWER_HALO, FIRST_OWN, LAST_OWN, UPPER_HALO = 0, 1, 2, 3


def split_planes(nk: int, parts: int) -> list[tuple[int, int]]:
    """(z0, nkl) of `parts` slabs covering nk planes: even sizes, as equal as
    possible, larger slabs first."""
    if nk % 2 or parts < 1 or nk < 2 * parts:
        raise ValueError(f"cannot split {nk} planes into {parts} even slabs")
    base, extra = divmod(nk // 2, parts)
    out, z0 = [], 0
    for r in range(parts):
        nkl = 2 * (base + (1 if r < extra else 0))
        out.append((z0, nkl))
        z0 += nkl
    return out


class SlabLattice(Lattice):
    """Global planes z0 .. z0+nkl-1 of an ni x nj x nk lattice, with halos."""

    def __init__(self, ni: int, nj: int, nk: int, z0: int, nkl: int, boundary: str = "open"):
        if boundary not in ("open", "periodic"):
            raise ValueError("boundary must be 'open' or 'periodic'")
        self._L = _lib.load()
        self.ni, self.nj, self.nk = int(ni), int(nj), int(nkl)
        self.nk_global, self.z0 = int(nk), int(z0)
        self.boundary = boundary
        h = ct.c_void_p()
        check(self._L.chll_lattice_create_slab(self.ni, self.nj, self.nk_global, self.z0, self.nk,
                                               _lib.CHLL_PERIODIC if boundary == "periodic"
                                               else _lib.CHLL_OPEN, ct.byref(h)))
        self._h = h

    def plane(self, colour: int, which: int) -> tuple[int, int]:
        """(device address, bytes) of one colour's plane (LOWER_HALO ... UPPER_HALO)."""
        p, n = ct.c_void_p(), ct.c_int64()
        check(self._L.chll_lattice_slab_plane(self._h, int(colour), int(which), ct.byref(p),
                                              ct.byref(n)))
        return p.value, n.value

    def counters(self) -> int:
        """Device address of the pass counters {director accepts, flips} (2 x uint64)."""
        p = ct.c_void_p()
        check(self._L.chll_lattice_counters(self._h, ct.byref(p)))
        return p.value

    def control_update(self, code: int) -> None:
        check(self._L.chll_lattice_control_update(self._h, int(code)))


class _DeviceArray:
    """A device address as a __cuda_array_interface__ object (zero-copy view)."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


def _plane_tensor(slab: SlabLattice, colour: int, which: int):
    import torch

    ptr, nbytes = slab.plane(colour, which)
    return torch.as_tensor(_DeviceArray(ptr, nbytes // 4, "<f4"), device="cuda")


def _counter_tensor(slab: SlabLattice):
    import torch

    return torch.as_tensor(_DeviceArray(slab.counters(), 2, "<i8"), device="cuda")


class LocalHalo:
    """Halo exchange and count sums for slabs held by this process, ordered on
    the current CUDA stream (the slabs must use the same stream)."""

    def __init__(self, slabs: list[SlabLattice]):
        self.slabs = list(slabs)
        self.periodic = self.slabs[0].boundary == "periodic"
        self._planes = [{(c, w): _plane_tensor(s, c, w) for c in (0, 1) for w in range(4)}
                        for s in self.slabs]
        self._counts = [_counter_tensor(s) for s in self.slabs]

    def exchange(self, colour: int) -> None:
        n = len(self.slabs)
        for r in range(n):
            up = r + 1 if r + 1 < n else (0 if self.periodic else None)
            if up is None:
                continue
            # my last own plane -> the next slab's lower halo, and back
            self._planes[up][(colour, LOWER_HALO)].copy_(self._planes[r][(colour, LAST_OWN)])
            self._planes[r][(colour, UPPER_HALO)].copy_(self._planes[up][(colour, FIRST_OWN)])

    def sum_counts(self, index: int) -> None:
        total = self._counts[0][index:index + 1].clone()
        for t in self._counts[1:]:
            total += t[index:index + 1]
        for t in self._counts:
            t[index:index + 1].copy_(total)


class TorchHalo:
    """Halo exchange and count sums with torch.distributed, one slab per rank.
    `planes(colour, which)` and `counts` are this rank's tensors (device tensors
    over the slab for NCCL; any tensors of the same sizes for gloo)."""

    def __init__(self, planes, counts, periodic: bool, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.periodic = periodic
        self.planes = planes
        self.counts = counts

    @classmethod
    def for_slab(cls, slab: SlabLattice, group=None):
        """The transport of `slab`, which from here on launches on the current
        CUDA stream: torch orders its NCCL operations after that stream's
        work, so passes and exchanges stay in order."""
        import torch

        slab.set_stream(torch.cuda.current_stream().cuda_stream)
        planes = {(c, w): _plane_tensor(slab, c, w) for c in (0, 1) for w in range(4)}
        return cls(lambda c, w: planes[(c, w)], _counter_tensor(slab),
                   slab.boundary == "periodic", group)

    def _neighbours(self):
        r, n = self.rank, self.world
        down = r - 1 if r > 0 else (n - 1 if self.periodic else None)
        up = r + 1 if r + 1 < n else (0 if self.periodic else None)
        return down, up

    def exchange(self, colour: int) -> None:
        dist = self.dist
        if self.world == 1:
            if self.periodic:  # a single periodic slab is its own neighbour
                self.planes(colour, LOWER_HALO).copy_(self.planes(colour, LAST_OWN))
                self.planes(colour, UPPER_HALO).copy_(self.planes(colour, FIRST_OWN))
            return
        down, up = self._neighbours()
        g = lambda r: dist.get_global_rank(self.group, r) if self.group is not None else r
        # Two phases, each one batch: messages between a pair of ranks match in
        # the order they are posted, and with two periodic ranks both
        # neighbours are the same rank.  Upward: my last own plane -> the
        # lower halo of the slab above; downward: my first own plane -> the
        # upper halo of the slab below.
        for send_which, send_to, recv_which, recv_from in (
                (LAST_OWN, up, LOWER_HALO, down), (FIRST_OWN, down, UPPER_HALO, up)):
            ops = []
            if send_to is not None:
                ops.append(dist.P2POp(dist.isend, self.planes(colour, send_which), g(send_to),
                                      self.group))
            if recv_from is not None:
                ops.append(dist.P2POp(dist.irecv, self.planes(colour, recv_which), g(recv_from),
                                      self.group))
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()

    def sum_counts(self, index: int) -> None:
        self.dist.all_reduce(self.counts[index:index + 1], group=self.group)


def sweep_slabs(slabs: list[SlabLattice], halo, cp, nsweeps: int, seed: int = 1,
                replica: int = 0) -> None:
    """nsweeps fused sweeps of the slabs held here, exchanging halos through
    `halo` (LocalHalo or TorchHalo); every slab ends with all trials done.
    The slabs must launch on the stream that is current while this runs (the
    halo copies and collectives are ordered on it)."""
    if nsweeps <= 0:
        return
    halo.exchange(0)
    halo.exchange(1)
    for s in range(nsweeps):
        for sl in slabs:
            sl.half_sweep(cp, FUSED_A if s else FUSED_A0, seed, replica)
        halo.exchange(0)
        if s:  # pass A closed the previous step's flips
            halo.sum_counts(1)
            for sl in slabs:
                sl.control_update(FUSED_A)
        for sl in slabs:
            sl.half_sweep(cp, FUSED_B, seed, replica)
        halo.exchange(1)
        halo.sum_counts(0)
        for sl in slabs:
            sl.control_update(FUSED_B)
    for sl in slabs:
        sl.half_sweep(cp, FUSED_F, seed, replica)
    halo.exchange(0)
    halo.sum_counts(1)
    for sl in slabs:
        sl.control_update(FUSED_F)


def slab_observables(rows: list[np.ndarray], nsites: int) -> dict:
    """Whole-lattice FP64 observables from the slabs' measurement rows (each
    row's raw sums cover the slab's own sites and the bonds they start)."""
    from .observables import nematic_S

    tot = np.sum([np.asarray(r, np.float64) for r in rows], axis=0)
    return {"energy": tot[_lib.ROW_ENERGY], "energy_per_site": tot[_lib.ROW_ENERGY] / nsites,
            "eta": tot[_lib.ROW_SUM_S] / nsites,
            "S": nematic_S(tot[_lib.ROW_QXX:_lib.ROW_QXX + 6], nsites),
            "etot_ref_sum": tot[_lib.ROW_ETOT_SUM]}
