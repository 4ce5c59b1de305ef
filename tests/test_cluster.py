"""The host side of a cluster shared by several ranks (edipic_b200.cluster), as world-size-2 gloo process groups on
the CPU: the listed int64 and FP64 buffers are summed in place over the ranks (exactly for int64), and each rank's id
range is disjoint and ends where the next rank's begins. Runs without a GPU."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from edipic_b200 import cluster


class FakeSim:
    """The two calls ClusterShare makes, over host buffers."""

    def __init__(self, rank):
        self.rho_e = np.arange(12, dtype=np.int64) * (1 << 33) + rank    # fixed-point values beyond 2^53 in sum
        self.rho_i = np.linspace(0.0, 1.0, 7) * (rank + 1)
        self.base = None

    def set_id_base(self, base, end=None):
        self.base = (base, end)

    def reduce_list(self):
        return [(self.rho_e.ctypes.data, self.rho_e.size, True), (self.rho_i.ctypes.data, self.rho_i.size, False)]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sim = FakeSim(rank)
        share = cluster.ClusterShare(sim, rank, world, device=False)
        share.reduce()
        out[rank] = (sim.base, sim.rho_e.copy(), sim.rho_i.copy())
    finally:
        dist.destroy_process_group()


def test_cluster_reduce_on_gloo():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    (b0, e0, i0), (b1, e1, i1) = out[0], out[1]
    want_e = 2 * (np.arange(12, dtype=np.int64) * (1 << 33)) + 1
    assert np.array_equal(e0, want_e) and np.array_equal(e1, want_e)
    assert np.allclose(i0, np.linspace(0.0, 1.0, 7) * 3) and np.array_equal(i0, i1)
    assert (b0, b1) == ((0, 1 << 31), (1 << 31, 1 << 32))
