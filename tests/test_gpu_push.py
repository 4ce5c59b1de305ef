"""One push of ADVANCE_ELECTRONS / ADVANCE_IONS on the device against the FP64 oracle on identical particles and
fields: positions within 1e-6 of a cell (mixed precision) or 1e-10 (FP64 path), velocities, wall / inner-object
absorption and hit counts, and the fused deposit against the oracle's CIC deposit of the same positions
(|drho| <= 2 * 2^-32 per contribution in fixed point)."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import (ELECTRONS, FIELD_ACC_EX, FIELD_ACC_EY, FIELD_EX, FIELD_EY, IONS, PREC_FP64, PREC_MIXED,
                         Simulation)
from gpu_common import contribution_bound, match_by_id, oracle_geom, periodic_dx, random_field, random_particles, small_deck

CASES = [("periodic", 0.0, 0.0), ("periodic", 86.6, 50.0), ("walled", 0.0, 0.0), ("walled", 86.6, 50.0)]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
@pytest.mark.parametrize("geometry,bx,by", CASES)
@pytest.mark.parametrize("species", [ELECTRONS, IONS])
@pytest.mark.parametrize("sort_every", [0, 4])
def test_push_matches_oracle(tmp_path, precision, geometry, bx, by, species, sort_every):
    if precision == PREC_FP64 and sort_every:
        pytest.skip("the FP64 path is unsorted")
    d = small_deck(tmp_path, geometry, bx=bx, by=by)
    with Simulation(d, precision=precision, sort_every=sort_every, fuse_collisions=False) as sim:
        p = sim.params
        n = 30000
        x, y, vx, vy, vz = random_particles(sim, n, seed=11 + species, precision=precision,
                                            vscale=0.05 if species == ELECTRONS else 0.002)
        if species == IONS:
            sim.upload_particles(ELECTRONS, x[:10], y[:10], vx[:10], vy[:10], vz[:10])
        ids = np.arange(n, dtype=np.uint32) * 3 + 7
        sim.upload_particles(species, x, y, vx, vy, vz, ids=ids)
        ex, ey = random_field(sim, precision=precision, amp=0.02 if species == ELECTRONS else 5.0)
        if species == ELECTRONS:
            sim.set_field(FIELD_EX, ex)
            sim.set_field(FIELD_EY, ey)
            sim.advance_electrons()
        else:
            sim.set_field(FIELD_ACC_EX, ex)
            sim.set_field(FIELD_ACC_EY, ey)
            sim.advance_ions()
        c = sim.counters()
        got = sim.download_particles(species)
        rho_gpu = sim.gather_electron_charge_density() if species == ELECTRONS else sim.gather_ion_charge_density()

    g = oracle_geom(sim)
    sp = pyoracle.Species(p.bx, p.by, p.bz, p.ez, 1 if species else 0, 0.5 * p.ion_charge[0] / p.ion_mass_me[0],
                          p.n_subcycles, p.ions_sense_b, p.ions_sense_ez)
    ps = pyoracle.ParticleSet(x, y, vx, vy, vz, ids=ids)
    hits = pyoracle.push(g, sp, ex, ey, ps)
    ref = ps.arrays()
    assert got["x"].size == ref["x"].size, (got["x"].size, ref["x"].size)
    ia, ib = match_by_id(got, ref)
    dxp = got["x"][ia] - ref["x"][ib]
    if sim.periodic:
        dxp = periodic_dx(dxp, p.ncx)
    tol = 1e-6 if precision == PREC_MIXED else 1e-10
    assert np.abs(dxp).max() < tol
    assert np.abs(got["y"][ia] - ref["y"][ib]).max() < tol
    vref = np.abs(np.stack([ref["vx"], ref["vy"], ref["vz"]])).max()
    for k in ("vx", "vy", "vz"):
        assert np.abs(got[k][ia] - ref[k][ib]).max() <= (2e-6 if precision == PREC_MIXED else 1e-12) * max(vref, 1e-3)
    hits_gpu = np.array(c.electron_hits[:8] if species == ELECTRONS else c.ion_hits[:8])
    assert np.array_equal(hits_gpu, hits), (hits_gpu, hits)
    assert hits.sum() > 0
    # deposit of the same (device) positions; the ion density is Qs-weighted
    pd = pyoracle.ParticleSet(got["x"], got["y"], got["vx"], got["vy"], got["vz"])
    w = 1.0 if species == ELECTRONS else float(p.ion_charge[0])
    rho_ref = pyoracle.deposit(g, pd, w)
    tol_rho = contribution_bound(sim, got["x"], got["y"]) if precision == PREC_MIXED else 1e-10
    assert np.all(np.abs(rho_gpu - rho_ref) <= tol_rho)
    assert abs(rho_gpu.sum() - rho_ref.sum()) < 1e-6
