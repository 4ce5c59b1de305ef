"""A cluster shared by two ranks against one context holding all the particles: each rank pushes half of the
particles over the whole grid, the densities are summed over the ranks after every step (gloo here: both ranks share
the one GPU this test gets, and gloo's sums are host-side, so no kernel waits on another), and after five steps of the
periodic FFT_X cycle (no collisions) the union of the ranks' particles equals the single context's particles bit for
bit in mixed precision (int64 fixed-point densities: the summed field is identical) and to rounding in FP64."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gpu_common import random_particles, small_deck

STEPS = 5


def _rows(d):
    o = np.argsort(d["id"])
    return np.stack([d[k][o] for k in ("x", "y", "vx", "vy", "vz")], axis=1), d["id"][o]


def _worker(rank, world, port, deck, precision, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from edipic_b200 import ELECTRONS, IONS, Simulation, cluster
    try:
        with Simulation(deck, precision=precision, sort_every=4, fuse_collisions=False) as sim:
            share = cluster.ClusterShare(sim, rank, world, blocking=True)
            n = 40000
            e = random_particles(sim, n, seed=1, precision=precision)
            i = random_particles(sim, n, seed=2, precision=precision, vscale=0.002)
            ids = np.arange(n, dtype=np.uint32)
            sim.upload_particles(ELECTRONS, *[a[rank::world] for a in e], ids=ids[rank::world])
            sim.upload_particles(IONS, *[a[rank::world] for a in i], ids=ids[rank::world])
            share.reduce()
            share.step(STEPS)
            out[rank] = [sim.download_particles(s) for s in (ELECTRONS, IONS)]
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_two_ranks_equal_one_context(tmp_path, precision):
    from edipic_b200 import ELECTRONS, IONS, PREC_FP64, PREC_MIXED, Simulation
    prec = PREC_MIXED if precision == "mixed" else PREC_FP64
    deck = small_deck(tmp_path, "periodic", collisions=False)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_worker, args=(2, port, deck, prec, out), nprocs=2, start_method="spawn", join=True)
    with Simulation(deck, precision=prec, sort_every=4, fuse_collisions=False) as sim:
        n = 40000
        ids = np.arange(n, dtype=np.uint32)
        sim.upload_particles(ELECTRONS, *random_particles(sim, n, seed=1, precision=prec), ids=ids)
        sim.upload_particles(IONS, *random_particles(sim, n, seed=2, precision=prec, vscale=0.002), ids=ids)
        sim.step(STEPS)
        ref = [sim.download_particles(s) for s in (ELECTRONS, IONS)]
    for s in range(2):
        both = {k: np.concatenate([out[0][s][k], out[1][s][k]]) for k in ref[s]}
        a, ia = _rows(both)
        b, ib = _rows(ref[s])
        assert np.array_equal(ia, ib)
        if prec == PREC_MIXED:
            assert np.array_equal(a, b)
        else:
            assert np.abs(a - b).max() < 1e-9
