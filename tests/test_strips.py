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

from edipic_b200.strips import REC, exchange_records, frames, partition, shift, split_particles


def test_partition_covers_the_columns():
    for ncx, n in ((64, 1), (64, 2), (64, 3), (1024, 7), (10, 10)):
        parts = partition(ncx, n)
        assert parts[0][0] == 0 and sum(w for _, w in parts) == ncx
        assert all(parts[k][0] + parts[k][1] == parts[k + 1][0] for k in range(n - 1))
        assert max(w for _, w in parts) - min(w for _, w in parts) <= 1
    with pytest.raises(ValueError):
        partition(4, 5)


@pytest.mark.parametrize("periodic", [True, False])
def test_owner_and_local_position(periodic):
    ncx, ghost = 64, 4
    parts = partition(ncx, 3)   # 22, 21, 21
    fr = frames(parts, ghost, periodic)
    if not periodic:   # the walls of the domain take no ghost columns
        assert fr[0][0] == 0 and fr[2][1] == 0 and fr[1] == (ghost, ghost, 22 - ghost)
    x = np.array([0.0, 21.999, 22.0, 42.5, 43.0, 63.75] + ([] if periodic else [64.0]))
    owner, local = split_particles(x, parts, [f[2] for f in fr])
    assert list(owner) == [0, 0, 1, 1, 2, 2] + ([] if periodic else [2])
    for o, xl, xg in zip(owner, local, x):
        x0, own = parts[o]
        gl = fr[o][0]
        assert gl <= xl <= gl + own and xl == xg - fr[o][2]


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_shifts_carry_ghost_particles_to_the_owner(n, periodic):
    """A particle in a ghost column of strip r, shifted as it is sent, lands in its neighbour's own columns at the
    same global position."""
    ncx, ghost = 60, 3
    parts = partition(ncx, n)
    fr = frames(parts, ghost, periodic)
    for r, (x0, own) in enumerate(parts):
        gl, gr, xf = fr[r]
        cases = [(0.25, "left"), (gl - 0.5, "left")] if gl else []
        cases += [(gl + own + 0.5, "right"), (gl + own + gr - 0.25, "right")] if gr else []
        for xl, side in cases:
            xg = (xf + xl) % ncx
            q = (r - 1) % n if side == "left" else (r + 1) % n
            wrap = (-1 if r == 0 else 0) if side == "left" else (1 if r == n - 1 else 0)
            x_new = xl + shift(xf, fr[q][2], wrap, ncx)
            qx0, qown = parts[q]
            assert fr[q][0] <= x_new < fr[q][0] + qown
            assert abs((fr[q][2] + x_new) % ncx - xg) < 1e-12


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
