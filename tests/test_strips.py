"""Host logic of the x strips without a GPU: the partition of the columns, the owner and local position of every
particle, the shifts that carry a ghost-column particle into its neighbour's columns, and the record exchange
between neighbouring ranks over gloo (two and three ranks on the CPU)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from edipic_b200.strips import REC, exchange_records, partition, split_particles


def test_partition_covers_the_columns():
    for ncx, n in ((64, 1), (64, 2), (64, 3), (1024, 7), (10, 10)):
        parts = partition(ncx, n)
        assert parts[0][0] == 0 and sum(w for _, w in parts) == ncx
        assert all(parts[k][0] + parts[k][1] == parts[k + 1][0] for k in range(n - 1))
        assert max(w for _, w in parts) - min(w for _, w in parts) <= 1
    with pytest.raises(ValueError):
        partition(4, 5)


def test_owner_and_local_position():
    ncx, ghost = 64, 4
    parts = partition(ncx, 3)   # 22, 21, 21
    x = np.array([0.0, 21.999, 22.0, 42.5, 43.0, 63.75])
    owner, local = split_particles(x, ncx, parts, ghost)
    assert list(owner) == [0, 0, 1, 1, 2, 2]
    for o, xl, xg in zip(owner, local, x):
        x0, own = parts[o]
        assert ghost <= xl < ghost + own and xl == xg - (x0 - ghost)


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_shifts_carry_ghost_particles_to_the_owner(n):
    """A particle in a ghost column of strip r, shifted as it is sent, lands in its neighbour's own columns at the
    same global (periodic) position."""
    ncx, ghost = 60, 3
    parts = partition(ncx, n)
    for r, (x0, own) in enumerate(parts):
        left_own = parts[(r - 1) % n][1]
        for xl, side in ((0.25, "left"), (ghost - 0.5, "left"), (ghost + own + 0.5, "right"),
                         (own + 2 * ghost - 0.25, "right")):
            xg = (x0 - ghost + xl) % ncx
            q = (r - 1) % n if side == "left" else (r + 1) % n
            x_new = xl + (left_own if side == "left" else -own)
            qx0, qown = parts[q]
            assert ghost <= x_new < ghost + qown
            assert abs((qx0 - ghost + x_new) % ncx - xg) < 1e-12


def _exchange_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        left = torch.full((rank + 1, REC), float(10 * rank + 1), dtype=torch.float64)    # to rank - 1
        right = torch.full((2 * rank + 3, REC), float(10 * rank + 2), dtype=torch.float64)   # to rank + 1
        fl, fr = exchange_records(left, right, rank, world)
        out[rank] = (fl.numpy().copy(), fr.numpy().copy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_records_between_neighbours(world):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_exchange_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        fl, fr = out[r]
        lo, hi = (r - 1) % world, (r + 1) % world
        # from the left neighbour: what it sent right; from the right neighbour: what it sent left
        assert fl.shape == (2 * lo + 3, REC) and np.all(fl == 10 * lo + 2)
        assert fr.shape == (hi + 1, REC) and np.all(fr == 10 * hi + 1)
