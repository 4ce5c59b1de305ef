"""A run saved to a checkpoint in the reference's layouts and continued in a fresh context: the particles come back
exactly (positions, velocities, tags; periodic overlap-cell positions folded), the step counter resumes at the saved
T_cntr, and two further steps without collisions give the same particles as the run that was not interrupted: bit
for bit with the FFT_X solve and the fixed-point deposit (the order of the particles does not matter), to rounding
otherwise."""
import os

import numpy as np
import pytest

from edipic_b200 import ELECTRONS, IONS, PREC_FP64, PREC_MIXED, Simulation, checkpoints
from gpu_common import random_particles, small_deck


def rows(d):
    a = np.stack([d["x"], d["y"], d["vx"], d["vy"], d["vz"], d["tag"].astype(np.float64)], axis=1)
    return a[np.lexsort(a.T[::-1])]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
@pytest.mark.parametrize("geometry", ["periodic", "walled"])
@pytest.mark.parametrize("fmt,nprocs", [("posix", 3), ("mpiio", 2)])
def test_checkpoint_restart(tmp_path, precision, geometry, fmt, nprocs):
    d = small_deck(tmp_path / "deck", geometry, collisions=False)
    root = str(tmp_path / "run")
    os.makedirs(root)
    n = 40000
    with Simulation(d, precision=precision, sort_every=4 if precision == PREC_MIXED else 0) as a:
        x, y, vx, vy, vz = random_particles(a, n, seed=3, precision=precision)
        tags = np.arange(n, dtype=np.int32) % 5
        a.upload_particles(ELECTRONS, x, y, vx, vy, vz, tag=tags)
        a.upload_particles(IONS, x, y, 0.01 * vx, 0.01 * vy, 0.01 * vz, tag=tags)
        a.set_step(37)
        a.step(3)   # a sorted state with dead slots
        t = int(a.counters().step)
        assert t == 40
        checkpoints.save_checkpoint(a, root, nprocs=nprocs, fmt=fmt, seed=11)
        before = [a.download_particles(s) for s in (ELECTRONS, IONS)]
        a.step(2)
        after_a = [a.download_particles(s) for s in (ELECTRONS, IONS)]
    with Simulation(d, precision=precision, sort_every=4 if precision == PREC_MIXED else 0) as b:
        loaded = checkpoints.load_checkpoint(b, t, root)
        assert len(loaded) == nprocs and int(b.counters().step) == t
        assert sum(len(r.electrons) for r in loaded) == len(before[0]["x"])
        for s, ref in zip((ELECTRONS, IONS), before):
            assert np.array_equal(rows(b.download_particles(s)), rows(ref))
        b.step(2)
        after_b = [b.download_particles(s) for s in (ELECTRONS, IONS)]
    for pa, pb in zip(after_a, after_b):
        ra, rb = rows(pa), rows(pb)
        assert ra.shape == rb.shape
        if precision == PREC_MIXED and geometry == "periodic":
            assert np.array_equal(ra, rb)
        else:
            # FP64 atomics sum the density in another order; the walled CG solve starts from the previous potential
            # in the uninterrupted run and from zero after the restart (a checkpoint holds no potential), so the
            # fields agree to the CG tolerance
            assert np.abs(ra - rb).max() < (1e-9 if geometry == "periodic" else 1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("fmt,nprocs", [("posix", 2), ("mpiio", 3)])
def test_checkpoint_dielectric_surface_charge(tmp_path, fmt, nprocs):
    """The outline charge of a dielectric inner object travels in rank 0's surface-charge block, in the order of the
    object's boundary nodes."""
    from edipic_b200 import FIELD_SURFACE_CHARGE
    diel = (30, 12, 40, 26, 0.0, 3.0)
    d = small_deck(tmp_path / "deck", "walled", inner=[diel], collisions=False)
    root = str(tmp_path / "run")
    os.makedirs(root)
    with Simulation(d, precision=PREC_MIXED, sort_every=0) as a:
        x, y, vx, vy, vz = random_particles(a, 5000, seed=9)
        a.upload_particles(ELECTRONS, x, y, vx, vy, vz)
        a.upload_particles(IONS, x, y, 0.01 * vx, 0.01 * vy, 0.01 * vz)
        surf = np.zeros((a.ny_ref, a.nx_ref))
        for (i, j) in checkpoints.outline_nodes(*diel[:4]):
            surf[j, i] = 0.25 * i - 0.5 * j
        a.set_field(FIELD_SURFACE_CHARGE, surf)
        a.set_step(5)
        checkpoints.save_checkpoint(a, root, nprocs=nprocs, fmt=fmt)
    with Simulation(d, precision=PREC_MIXED, sort_every=0) as b:
        ranks = checkpoints.load_checkpoint(b, 5, root)
        assert len(ranks[0].surf) == 2 * (10 + 14) and all(len(r.surf) == 0 for r in ranks[1:])
        assert np.abs(b.field(FIELD_SURFACE_CHARGE) - surf).max() < 1e-9
