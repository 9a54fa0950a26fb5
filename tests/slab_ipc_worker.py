"""One rank of the multi-process slab test (tests/test_slab_ipc_gpu.py): a
slab of a lattice on GPU 0 whose passes write its boundary planes into the
neighbouring ranks' halos through CUDA IPC mappings (TorchPeerHalo over
gloo).  Writes its final own planes and control block to OUT/rank<r>.npz.

usage: slab_ipc_worker.py RANK WORLD PORT OUT NI NJ NK BOUNDARY NSWEEPS"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    rank, world, port = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3])
    out = sys.argv[4]
    ni, nj, nk = (int(a) for a in sys.argv[5:8])
    boundary, nsw = sys.argv[8], int(sys.argv[9])
    import torch
    import torch.distributed as dist

    from chllmodel_b200.lattice import coupling
    from chllmodel_b200.slab import SlabLattice, TorchPeerHalo, split_planes, sweep_slabs

    torch.cuda.set_device(0)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        z0, nkl = split_planes(nk, world)[rank]
        sl = SlabLattice(ni, nj, nk, z0, nkl, boundary=boundary)
        sl.set_stream(torch.cuda.current_stream().cuda_stream)
        sl.init_random(31, 2)
        sl.set_control(0.15, step=1)
        halo = TorchPeerHalo.for_slab(sl)
        cp = coupling(0.6, 1.0, 0.2, 1.1)
        sweep_slabs([sl], halo, cp, 3, seed=5, replica=2)
        sweep_slabs([sl], halo, cp, nsw - 3, seed=5, replica=2)
        torch.cuda.synchronize()
        state = sl.download_f4()
        ctl = sl.control()
        halo.close()
        np.savez(os.path.join(out, f"rank{rank}.npz"), state=state,
                 ctl=np.array([ctl["d"], ctl["step"], ctl["paccept"], ctl["faccept"]]))
        sl.close()
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
