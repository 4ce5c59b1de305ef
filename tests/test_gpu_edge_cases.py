"""Edge cases of the device cycle against the oracle: empty species (the cycle, diagnostics and downloads on zero
particles), a ragged particle count with particles exactly on cell edges and on the walls, one particle followed for
many steps in the magnetised cfg1 field, and the largest FFT_X grid (4096 columns)."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import (ELECTRONS, FIELD_EX, FIELD_EY, FIELD_PHI, FIELD_RHO_TOTAL, IONS, PREC_FP64, PREC_MIXED,
                         Simulation)
from gpu_common import match_by_id, oracle_geom, periodic_dx, random_field, random_particles, small_deck


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
@pytest.mark.parametrize("geometry", ["periodic", "walled"])
def test_empty_species(tmp_path, precision, geometry):
    d = small_deck(tmp_path, geometry, wall_potentials={2: 30.0, 4: -10.0})
    with Simulation(d, precision=precision, sort_every=4) as sim:
        z = np.zeros(0)
        sim.upload_particles(ELECTRONS, z, z, z, z, z)
        sim.upload_particles(IONS, z, z, z, z, z)
        sim.step(5)
        c = sim.counters()
        rho = sim.field(FIELD_RHO_TOTAL)
        phi = sim.field(FIELD_PHI)
        m = sim.collect_moments(ELECTRONS)
        v1, v2, sk = sim.calculate_vdf(IONS, (2, 2), 4, 10, True)
        e = sim.download_particles(ELECTRONS)
        p = sim.params
    assert list(c.n_particles[:2]) == [0, 0] and sum(c.electron_hits) == 0
    assert not rho.any() and not m.any() and not v1.any() and not v2.any() and sk == 0
    assert e["x"].size == 0
    # no charge: phi is the Laplace solution of the electrode potentials (a linear profile across the periodic gap;
    # the CG solve of the oracle for the walls and the -100 V object, to the cycle's relative residual of 1e-8)
    if geometry == "periodic":
        j = np.arange(p.ncy + 1)[:, None]
        ref = p.wall_phi_const[0] + (p.wall_phi_const[1] - p.wall_phi_const[0]) * j / p.ncy + 0 * phi
        tol = 1e-9
    else:
        ref, _, _ = pyoracle.cg_solve(oracle_geom(sim), np.zeros_like(phi), list(p.wall_phi_const),
                                      [p.inner_phi[0]], rtol=1e-13)
        tol = 1e-5
        for a in (phi, ref):   # corner nodes touch no unknown; which wall owns them is a convention
            a[[0, 0, -1, -1], [0, -1, 0, -1]] = 0.0
    assert np.abs(phi - ref).max() <= tol * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
@pytest.mark.parametrize("geometry", ["periodic", "walled"])
def test_ragged_count_and_edge_positions(tmp_path, precision, geometry):
    d = small_deck(tmp_path, geometry, bx=86.6, by=50.0, **({} if geometry == "periodic" else {"inner": False}))
    with Simulation(d, precision=precision, sort_every=4, fuse_collisions=False) as sim:
        p = sim.params
        n = 4097   # not a multiple of the 4-particle groups
        x, y, vx, vy, vz = random_particles(sim, n, seed=21, precision=precision)
        xmax = float(p.ncx) if geometry == "walled" else float(p.ncx) - 0.5
        edge = [(0.0, 0.0), (0.0, 7.0), (5.0, 0.0), (5.0, float(p.ncy)), (xmax, 3.0), (13.0, 9.0), (13.0, 9.5),
                (2.0, float(p.ncy) - 0.5)]
        for k, (ex_, ey_) in enumerate(edge):
            x[k], y[k] = ex_, ey_
        vx[:len(edge)] *= 0.1
        ids = np.arange(n, dtype=np.uint32) + 11
        sim.upload_particles(ELECTRONS, x, y, vx, vy, vz, ids=ids)
        ex, ey = random_field(sim, precision=precision)
        sim.set_field(FIELD_EX, ex)
        sim.set_field(FIELD_EY, ey)
        sim.advance_electrons()
        c = sim.counters()
        got = sim.download_particles(ELECTRONS)
    g = oracle_geom(sim)
    sp = pyoracle.Species(p.bx, p.by, p.bz, p.ez, 0, 0.0, p.n_subcycles, p.ions_sense_b, p.ions_sense_ez)
    ps = pyoracle.ParticleSet(x, y, vx, vy, vz, ids=ids)
    hits = pyoracle.push(g, sp, ex, ey, ps)
    ref = ps.arrays()
    assert got["x"].size == ref["x"].size
    assert np.array_equal(np.array(c.electron_hits[:8]), hits)
    ia, ib = match_by_id(got, ref)
    dxp = got["x"][ia] - ref["x"][ib]
    if sim.periodic:
        dxp = periodic_dx(dxp, p.ncx)
    tol = 1e-6 if precision == PREC_MIXED else 1e-10
    assert np.abs(dxp).max() < tol and np.abs(got["y"][ia] - ref["y"][ib]).max() < tol


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_one_particle_many_steps(tmp_path, precision):
    """One electron gyrating in the 10 mT field of cfg1 through a fixed E for 200 pushes."""
    d = small_deck(tmp_path, "periodic", bx=86.6, by=50.0)
    with Simulation(d, precision=precision, sort_every=0, fuse_collisions=False) as sim:
        p = sim.params
        x, y, vx, vy, vz = (np.array([v]) for v in (20.25, 24.5, 0.15, -0.05, 0.1))
        if precision == PREC_MIXED:
            vx, vy, vz = (a.astype(np.float32).astype(np.float64) for a in (vx, vy, vz))
        sim.upload_particles(ELECTRONS, x, y, vx, vy, vz)
        ex, ey = random_field(sim, precision=precision, amp=0.002)
        track = []
        for _ in range(200):
            sim.set_field(FIELD_EX, ex)
            sim.set_field(FIELD_EY, ey)
            sim.advance_electrons()
            e = sim.download_particles(ELECTRONS)
            track.append([e["x"][0], e["y"][0], e["vx"][0], e["vy"][0], e["vz"][0]])
    g = oracle_geom(sim)
    sp = pyoracle.Species(p.bx, p.by, p.bz, p.ez, 0, 0.0, p.n_subcycles, p.ions_sense_b, p.ions_sense_ez)
    ps = pyoracle.ParticleSet(x, y, vx, vy, vz)
    ref = []
    for _ in range(200):
        pyoracle.push(g, sp, ex, ey, ps)
        a = ps.arrays()
        ref.append([a["x"][0], a["y"][0], a["vx"][0], a["vy"][0], a["vz"][0]])
    t, r = np.array(track), np.array(ref)
    dx = periodic_dx(t[:, 0] - r[:, 0], p.ncx)
    # FP32 state drifts from the FP64 one by rounding each step; FP64 stays at rounding level
    tol = 2e-4 if precision == PREC_MIXED else 1e-9
    assert np.abs(dx).max() < tol and np.abs(t[:, 1] - r[:, 1]).max() < tol
    assert np.abs(t[:, 2:] - r[:, 2:]).max() < tol


@pytest.mark.gpu
def test_largest_fftx_grid(tmp_path):
    d = small_deck(tmp_path, "periodic", ncx=4096, ncy=12, ppc=1, wall_potentials={2: 20.0, 4: -5.0})
    with Simulation(d, precision=PREC_FP64, sort_every=0) as sim:
        p = sim.params
        x, y, vx, vy, vz = random_particles(sim, 200000, seed=5, precision=PREC_FP64)
        sim.upload_particles(ELECTRONS, x, y, vx, vy, vz)
        sim.upload_particles(IONS, x[::2], y[::2], 0 * vx[::2], 0 * vy[::2], 0 * vz[::2])
        phi = sim.solve_poisson_fftx_linsysy(want_phi=True)
        rho = sim.field(FIELD_RHO_TOTAL)
    ref = pyoracle.fftx_solve(oracle_geom(sim), rho, p.wall_phi_const[0], p.wall_phi_const[1])
    assert np.abs(phi - ref).max() <= 1e-9 * np.abs(ref).max()
