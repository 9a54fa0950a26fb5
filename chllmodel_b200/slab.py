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
with host tensors) for one slab per rank.  ``PeerHalo`` (one process) and
``TorchPeerHalo`` (one slab per rank, CUDA IPC) move no planes between passes:
the passes themselves store the boundary planes into the neighbours' halos.
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


def neighbours(r: int, n: int, periodic: bool) -> tuple[int | None, int | None]:
    """(slab below, slab above) of slab r of n along z; None past an open end.
    A single periodic slab is its own neighbour on both sides."""
    down = r - 1 if r > 0 else (n - 1 if periodic else None)
    up = r + 1 if r + 1 < n else (0 if periodic else None)
    return down, up


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

    def set_peers(self, lower=(None, None), upper=(None, None)) -> None:
        """From now on every pass of colour c also writes this slab's first own
        plane to the device address lower[c] and its last own plane to
        upper[c]: the upper halo of the slab below and the lower halo of the
        slab above (None: no neighbour on that side)."""
        v = lambda a: ct.c_void_p(a) if a else None
        check(self._L.chll_lattice_slab_set_peers(self._h, v(lower[0]), v(lower[1]), v(upper[0]),
                                                  v(upper[1])))

    def push(self, colour: int) -> None:
        """Copies the own boundary planes of one colour to the peers."""
        check(self._L.chll_lattice_slab_push(self._h, int(colour)))

    def ipc_handle(self) -> tuple[bytes, int]:
        """(64-byte CUDA IPC handle of the lattice allocation, its base address)."""
        buf = ct.create_string_buffer(64)
        base = ct.c_uint64()
        check(self._L.chll_lattice_ipc_handle(self._h, buf, ct.byref(base)))
        return buf.raw, base.value


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
            up = neighbours(r, n, self.periodic)[1]
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


class PeerHalo(LocalHalo):
    """Slabs held by this process whose passes write their boundary planes
    straight into the neighbouring slabs' halo planes (set_peers), so no copy
    is left between passes: the single stream orders the passes.  Count sums
    as LocalHalo."""

    def __init__(self, slabs: list[SlabLattice]):
        super().__init__(slabs)
        n = len(self.slabs)
        for r, sl in enumerate(self.slabs):
            down, up = neighbours(r, n, self.periodic)
            lower = [self.slabs[down].plane(c, UPPER_HALO)[0] if down is not None else None
                     for c in (0, 1)]
            upper = [self.slabs[up].plane(c, LOWER_HALO)[0] if up is not None else None
                     for c in (0, 1)]
            sl.set_peers(lower, upper)

    def prime(self, colour: int) -> None:
        for sl in self.slabs:
            sl.push(colour)

    def exchange(self, colour: int) -> None:
        pass  # written by the passes themselves


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
        slab.set_stream(_lib.torch_stream_handle())
        planes = {(c, w): _plane_tensor(slab, c, w) for c in (0, 1) for w in range(4)}
        return cls(lambda c, w: planes[(c, w)], _counter_tensor(slab),
                   slab.boundary == "periodic", group)

    def _neighbours(self):
        return neighbours(self.rank, self.world, self.periodic)

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


class TorchPeerHalo(TorchHalo):
    """One slab per rank, halos written inside the passes over peer memory.

    Each rank maps its neighbours' lattice allocations (CUDA IPC,
    chll_lattice_ipc_handle / chll_ipc_open, exchanged with all_gather) and
    sets their halo planes as its slab's peers: a pass of colour c writes the
    slab's boundary planes of colour c into the neighbours' halos as it
    updates them (one 256-bit store per boundary unit, over NVLink between
    GPUs).  Between passes only the ordering is left, and it comes from the
    collectives that follow every pass: the count all-reduce, or a
    one-element all-reduce after a pass that closes no count (exchange()).
    Every rank's next pass starts after every rank's previous pass, so a
    halo is never written while it is read.  With NCCL the collectives are
    ordered on the current stream; with gloo (tests: processes sharing one
    GPU) the device is synchronised around them.  No kernel waits on
    another GPU."""

    def __init__(self, slab: SlabLattice, group=None):
        import torch
        import torch.distributed as dist

        slab.set_stream(_lib.torch_stream_handle())
        super().__init__(None, _counter_tensor(slab), slab.boundary == "periodic", group)
        self.slab = slab
        self.gloo = dist.get_backend(group) == "gloo"
        handle, base = slab.ipc_handle()
        offs = {(c, w): slab.plane(c, w)[0] - base for c in (0, 1)
                for w in (LOWER_HALO, UPPER_HALO)}
        info = [None] * self.world
        dist.all_gather_object(info, (handle, offs), group=group)
        down, up = self._neighbours()
        self._mapped = {}

        def base_of(r):
            if r == self.rank:
                return base
            if r not in self._mapped:
                p = ct.c_void_p()
                check(slab._L.chll_ipc_open(info[r][0], ct.byref(p)))
                self._mapped[r] = p.value
            return self._mapped[r]

        lower = [base_of(down) + info[down][1][(c, UPPER_HALO)] if down is not None else None
                 for c in (0, 1)]
        upper = [base_of(up) + info[up][1][(c, LOWER_HALO)] if up is not None else None
                 for c in (0, 1)]
        slab.set_peers(lower, upper)
        self._token = torch.zeros(1, dtype=torch.int64,
                                  device="cpu" if self.gloo else "cuda")

    @classmethod
    def for_slab(cls, slab: SlabLattice, group=None):
        return cls(slab, group)

    def _all_reduce(self, t) -> None:
        import torch

        if self.gloo:
            torch.cuda.current_stream().synchronize()
            host = t.cpu() if t.is_cuda else t
            self.dist.all_reduce(host, group=self.group)
            if t.is_cuda:
                t.copy_(host)
                torch.cuda.current_stream().synchronize()
        else:
            self.dist.all_reduce(t, group=self.group)

    def prime(self, colour: int) -> None:
        self._all_reduce(self._token)   # neighbours' previous passes are done
        self.slab.push(colour)
        self._all_reduce(self._token)   # and every halo is filled

    def exchange(self, colour: int) -> None:
        self._all_reduce(self._token)

    def sum_counts(self, index: int) -> None:
        self._all_reduce(self.counts[index:index + 1])

    def exchange_and_sum(self, colour: int, index: int) -> None:
        """After a pass that closes a count: the count's all-reduce is a
        collective on the same stream after every rank's pass, so it orders
        the passes (and the halo stores in them) as the token would."""
        self.sum_counts(index)

    def close(self) -> None:
        """Unmaps the neighbours' allocations after the last pass; collective
        (every rank calls it before freeing its slab)."""
        import torch

        torch.cuda.current_stream().synchronize()
        self._all_reduce(self._token)   # no rank still writes into a mapped halo
        self.slab.set_peers()
        for p in self._mapped.values():
            check(self.slab._L.chll_ipc_close(ct.c_void_p(p)))
        self._mapped = {}
        torch.cuda.current_stream().synchronize()
        self._all_reduce(self._token)   # every mapping of this slab is gone before it is freed


def sweep_slabs(slabs: list[SlabLattice], halo, cp, nsweeps: int, seed: int = 1,
                replica: int = 0) -> None:
    """nsweeps fused sweeps of the slabs held here, exchanging halos through
    `halo` (LocalHalo, PeerHalo, TorchHalo or TorchPeerHalo); every slab ends
    with all trials done.  The slabs must launch on the stream that is
    current while this runs (the halo copies and collectives are ordered on
    it)."""
    if nsweeps <= 0:
        return
    prime = getattr(halo, "prime", halo.exchange)  # the halos' first fill
    # halo exchange plus the sum of the count the pass closed; a transport
    # whose exchange is only an ordering collective does both in one
    closing = getattr(halo, "exchange_and_sum", None)

    def close(colour: int, index: int) -> None:
        if closing is not None:
            closing(colour, index)
        else:
            halo.exchange(colour)
            halo.sum_counts(index)

    prime(0)
    prime(1)
    for s in range(nsweeps):
        for sl in slabs:
            sl.half_sweep(cp, FUSED_A if s else FUSED_A0, seed, replica)
        if s:  # pass A closed the previous step's flips
            close(0, 1)
            for sl in slabs:
                sl.control_update(FUSED_A)
        else:
            halo.exchange(0)
        for sl in slabs:
            sl.half_sweep(cp, FUSED_B, seed, replica)
        close(1, 0)
        for sl in slabs:
            sl.control_update(FUSED_B)
    for sl in slabs:
        sl.half_sweep(cp, FUSED_F, seed, replica)
    close(0, 1)
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
