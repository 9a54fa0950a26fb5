"""A lattice split over processes: one z-slab per rank, the ranks' passes
writing their boundary planes into the neighbouring ranks' halo planes
through CUDA IPC mappings (slab.TorchPeerHalo), with the count sums and the
ordering over gloo.  The ranks share the one GPU here, as separate
processes; no kernel waits on another, the host orders every pass through
the collectives.  The joined state and every rank's control block must
equal the whole lattice's after the same sweeps."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WORKER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "slab_ipc_worker.py")


@pytest.mark.parametrize("shape,boundary,world", [((12, 10, 12), "periodic", 2),
                                                  ((10, 8, 12), "open", 3),
                                                  ((8, 6, 8), "periodic", 1)])
def test_ipc_slabs_follow_the_whole_lattice(tmp_path, shape, boundary, world):
    from chllmodel_b200.lattice import Lattice, coupling

    nsw = 6
    whole = Lattice(*shape, boundary=boundary)
    whole.init_random(31, 2)
    whole.set_control(0.15, step=1)
    whole.sweep(coupling(0.6, 1.0, 0.2, 1.1), nsw, seed=5, replica=2)
    ref_state = whole.download_f4()
    ref_ctl = whole.control()
    whole.close()

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [subprocess.Popen([sys.executable, WORKER, str(r), str(world), str(port),
                               str(tmp_path), *map(str, shape), boundary, str(nsw)],
                              stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
             for r in range(world)]
    outs = []
    try:
        for p in procs:
            outs.append(p.communicate(timeout=240)[0].decode(errors="replace"))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    for p, o in zip(procs, outs):
        assert p.returncode == 0, o[-3000:]
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    state = np.concatenate([d["state"] for d in parts], axis=0)
    assert np.array_equal(state, ref_state)
    want = np.array([ref_ctl["d"], ref_ctl["step"], ref_ctl["paccept"], ref_ctl["faccept"]])
    for d in parts:
        assert np.array_equal(d["ctl"], want)
