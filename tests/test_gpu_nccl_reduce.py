"""The NCCL path of the cluster sum on the library's own buffers and stream, on the one GPU this test gets: a
one-rank NCCL group sums the listed int64 densities in place (a sum over one rank leaves them unchanged), ordered on
the library's stream, and the cycle continues from them."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gpu_common import random_particles, small_deck


def _worker(rank, port, deck, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    from edipic_b200 import ELECTRONS, FIELD_RHO_TOTAL, IONS, Simulation, cluster
    try:
        with Simulation(deck, sort_every=4) as sim:
            n = 30000
            sim.upload_particles(ELECTRONS, *random_particles(sim, n, seed=1))
            sim.upload_particles(IONS, *random_particles(sim, n, seed=2, vscale=0.002))
            entries = sim.reduce_list()
            before = [torch.as_tensor(cluster._Buffer(p, c, i, True), device="cuda").clone() for p, c, i in entries]
            cluster.allreduce_buffers(entries, True, None, sim.stream())
            sim.synchronize()
            after = [torch.as_tensor(cluster._Buffer(p, c, i, True), device="cuda") for p, c, i in entries]
            same = all(bool(torch.equal(a, b)) for a, b in zip(after, before))
            sim.step(2)
            entries2 = sim.reduce_list()
            cluster.allreduce_buffers(entries2, True, None, sim.stream())
            sim.step(1)
            rho = sim.field(FIELD_RHO_TOTAL)
            out["r"] = (len(entries), all(i for _, _, i in entries), same, len(entries2), bool(np.isfinite(rho).all()))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_nccl_sum_on_library_buffers(tmp_path):
    deck = small_deck(tmp_path, "periodic")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_worker, args=(port, deck, out), nprocs=1, start_method="spawn", join=True)
    n, ints, same, n2, finite = out["r"]
    assert n == 2 and ints and same and finite
    assert n2 == 2   # electrons every step, ions on their step
