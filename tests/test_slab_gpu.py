"""z-slabs on one GPU: a lattice split into slabs that exchange halo planes
between passes (LocalHalo) or write them into each other's halos during the
passes (PeerHalo) follows the whole lattice's chain bit for bit, and the
slabs' measurement rows add up to the whole lattice's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("transport", ["copies", "peer"])
@pytest.mark.parametrize("shape,boundary,parts", [((16, 12, 16), "periodic", 2),
                                                  ((16, 12, 16), "periodic", 4),
                                                  ((12, 10, 12), "open", 3),
                                                  ((9, 6, 10), "open", 2),
                                                  ((8, 8, 6), "periodic", 3),
                                                  ((8, 8, 6), "periodic", 1)])
def test_slabs_follow_the_whole_lattice(shape, boundary, parts, transport):
    """transport "copies": LocalHalo copies the boundary planes between
    passes; "peer": PeerHalo, the passes write them into the neighbours'
    halos themselves (one periodic slab is its own neighbour)."""
    import torch

    from chllmodel_b200.lattice import Lattice, coupling
    from chllmodel_b200.slab import LocalHalo, PeerHalo, SlabLattice, slab_observables, \
        split_planes, sweep_slabs

    ni, nj, nk = shape
    cp = coupling(0.6, 1.0, 0.2, 1.1)
    nsw = 7
    whole = Lattice(*shape, boundary=boundary)
    whole.init_random(31, 2)
    whole.set_control(0.15, step=1)
    whole.sweep(cp, nsw, seed=5, replica=2)
    ref_state = whole.download_f4()
    ref_ctl = whole.control()
    ref_row = whole.observe(cp)
    whole.close()

    s = torch.cuda.Stream()
    slabs = []
    for z0, nkl in split_planes(nk, parts):
        sl = SlabLattice(ni, nj, nk, z0, nkl, boundary=boundary)
        sl.set_stream(s.cuda_stream)
        sl.init_random(31, 2)
        sl.set_control(0.15, step=1)
        slabs.append(sl)
    with torch.cuda.stream(s):
        halo = LocalHalo(slabs) if transport == "copies" else PeerHalo(slabs)
        sweep_slabs(slabs, halo, cp, 4, seed=5, replica=2)
        sweep_slabs(slabs, halo, cp, nsw - 4, seed=5, replica=2)
    s.synchronize()
    state = np.concatenate([sl.download_f4() for sl in slabs], axis=0)
    assert np.array_equal(state, ref_state)
    for sl in slabs:
        assert sl.control() == ref_ctl
    obs = slab_observables([sl.observe(cp) for sl in slabs], ni * nj * nk)
    assert obs["energy"] == pytest.approx(ref_row[5], rel=1e-12, abs=1e-9)
    assert obs["eta"] * ni * nj * nk == pytest.approx(ref_row[6], rel=1e-12)
    assert obs["etot_ref_sum"] == pytest.approx(ref_row[13], rel=1e-12, abs=1e-9)
    for sl in slabs:
        sl.close()


def test_slab_rejects_whole_lattice_calls():
    from chllmodel_b200 import _lib
    from chllmodel_b200.lattice import coupling
    from chllmodel_b200.slab import SlabLattice

    with pytest.raises(_lib.ChllError, match="even"):
        SlabLattice(8, 8, 8, 1, 2)
    sl = SlabLattice(8, 8, 8, 2, 4)
    with pytest.raises(_lib.ChllError, match="pass by pass"):
        sl.sweep(coupling(1.0, 1.0), 1)
    with pytest.raises(_lib.ChllError, match="fused passes"):
        sl.half_sweep(coupling(1.0, 1.0), 0)
    with pytest.raises(_lib.ChllError, match="slab"):
        sl.quench(coupling(1.0, 1.0), 0.1, 1)
    with pytest.raises(_lib.ChllError, match="resident"):
        sl.set_kernel("resident")
    sl.close()


def test_torch_halo_with_one_nccl_rank():
    """TorchHalo.for_slab (tensor views over the slab's device planes and
    counters, NCCL all-reduce of the counts) with a one-rank group: one
    periodic slab holding the whole lattice is its own neighbour and follows
    the whole lattice's chain."""
    import os
    import socket

    import torch
    import torch.distributed as dist

    from chllmodel_b200.lattice import Lattice, coupling
    from chllmodel_b200.slab import SlabLattice, TorchHalo, sweep_slabs

    shape = (12, 10, 8)
    cp = coupling(0.7, 1.0, 0.1)
    whole = Lattice(*shape, boundary="periodic")
    whole.init_random(9)
    whole.set_control(0.2, step=1)
    whole.sweep(cp, 5, seed=3)
    ref = whole.download_f4(), whole.control()
    whole.close()

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1,
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        sl = SlabLattice(*shape, 0, shape[2], boundary="periodic")
        stream = torch.cuda.current_stream()
        sl.set_stream(stream.cuda_stream)
        sl.init_random(9)
        sl.set_control(0.2, step=1)
        sweep_slabs([sl], TorchHalo.for_slab(sl), cp, 5, seed=3)
        torch.cuda.synchronize()
        assert np.array_equal(sl.download_f4(), ref[0])
        assert sl.control() == ref[1]
        sl.close()
    finally:
        dist.destroy_process_group()


def test_slab_peers_are_checked():
    """set_peers takes 32-byte aligned device addresses of a slab only: a
    misaligned or host address, or a whole lattice, is refused before any
    pass can store to it."""
    import ctypes as ct

    import numpy as np

    from chllmodel_b200 import _lib
    from chllmodel_b200.lattice import Lattice
    from chllmodel_b200.slab import LOWER_HALO, UPPER_HALO, SlabLattice

    a = SlabLattice(8, 8, 8, 0, 4, boundary="periodic")
    b = SlabLattice(8, 8, 8, 4, 4, boundary="periodic")
    good = b.plane(0, LOWER_HALO)[0]
    with pytest.raises(_lib.ChllError, match="32-byte aligned"):
        a.set_peers(upper=(good + 16, None))
    host = np.zeros(64, np.float32)
    host_aligned = (host.ctypes.data + 31) & ~31
    with pytest.raises(_lib.ChllError, match="device memory"):
        a.set_peers(upper=(host_aligned, None))
    a.set_peers(lower=(b.plane(0, UPPER_HALO)[0], b.plane(1, UPPER_HALO)[0]),
                upper=(good, b.plane(1, LOWER_HALO)[0]))
    a.set_peers()
    whole = Lattice(8, 8, 8)
    L = _lib.load()
    rc = L.chll_lattice_slab_set_peers(whole._h, ct.c_void_p(good), None, None, None)
    assert rc == _lib.CHLL_EINVAL and b"not a slab" in L.chll_last_error()
    for x in (a, b, whole):
        x.close()


def test_torch_peer_halo_with_one_nccl_rank():
    """TorchPeerHalo on its NCCL path (the collectives ordered on the stream)
    with a one-rank group: one periodic slab is its own neighbour, so its
    passes store their boundary planes into their own halos, and it follows
    the whole lattice's chain."""
    import os
    import socket

    import torch
    import torch.distributed as dist

    from chllmodel_b200.lattice import Lattice, coupling
    from chllmodel_b200.slab import SlabLattice, TorchPeerHalo, sweep_slabs

    shape = (12, 10, 8)
    cp = coupling(0.7, 1.0, 0.1)
    whole = Lattice(*shape, boundary="periodic")
    whole.init_random(9)
    whole.set_control(0.2, step=1)
    whole.sweep(cp, 5, seed=3)
    ref = whole.download_f4(), whole.control()
    whole.close()

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1,
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        sl = SlabLattice(*shape, 0, shape[2], boundary="periodic")
        sl.init_random(9)
        sl.set_control(0.2, step=1)
        halo = TorchPeerHalo.for_slab(sl)
        sweep_slabs([sl], halo, cp, 2, seed=3)
        sweep_slabs([sl], halo, cp, 3, seed=3)
        torch.cuda.synchronize()
        assert np.array_equal(sl.download_f4(), ref[0])
        assert sl.control() == ref[1]
        halo.close()
        sl.close()
    finally:
        dist.destroy_process_group()
