"""COLLECT_ELECTRON_MOMENTS / COLLECT_ION_MOMENTS on the device against the oracle on identical particles and field:
the 13 normalised node grids (density with the wall factors, mean velocities, second moments, heat fluxes), for the
sorted mixed-precision layout (tile windows plus particles that left their window) and the FP64 path."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import ELECTRONS, FIELD_EX, FIELD_EY, IONS, PREC_FP64, PREC_MIXED, Simulation
from gpu_common import oracle_geom, random_field, random_particles, small_deck

NAMES = ["N", "VX", "VY", "VZ", "WX", "WY", "WZ", "VXVY", "VXVZ", "VYVZ", "QX", "QY", "QZ"]


@pytest.mark.gpu
@pytest.mark.parametrize("precision,sort_every", [(PREC_MIXED, 4), (PREC_MIXED, 0), (PREC_FP64, 0)])
@pytest.mark.parametrize("geometry", ["periodic", "walled"])
@pytest.mark.parametrize("species", [ELECTRONS, IONS])
def test_moments_match_oracle(tmp_path, precision, sort_every, geometry, species):
    d = small_deck(tmp_path, geometry, bx=86.6, by=50.0)
    with Simulation(d, precision=precision, sort_every=sort_every, fuse_collisions=False) as sim:
        p = sim.params
        n = 60000
        x, y, vx, vy, vz = random_particles(sim, n, seed=31 + species, precision=precision,
                                            vscale=0.05 if species == ELECTRONS else 0.002)
        sim.upload_particles(ELECTRONS, x, y, vx, vy, vz)
        if species == IONS:
            sim.upload_particles(IONS, x, y, 0.04 * vx, 0.04 * vy, 0.04 * vz)
        ex, ey = random_field(sim, precision=precision, amp=0.02)
        sim.set_field(FIELD_EX, ex)
        sim.set_field(FIELD_EY, ey)
        sim.advance_electrons()   # particles leave their sorted tiles; the window and global paths both run
        ex2, ey2 = random_field(sim, precision=precision, amp=0.02, seed=9)
        sim.set_field(FIELD_EX, ex2)
        sim.set_field(FIELD_EY, ey2)
        got = sim.collect_moments(species).astype(np.float64)
        parts = sim.download_particles(species)
    g = oracle_geom(sim)
    sp = pyoracle.Species(p.bx, p.by, p.bz, p.ez, 1 if species else 0, 0.5 * p.ion_charge[0] / p.ion_mass_me[0],
                          p.n_subcycles, p.ions_sense_b, p.ions_sense_ez)
    ps = pyoracle.ParticleSet(parts["x"], parts["y"], parts["vx"], parts["vy"], parts["vz"])
    ref = pyoracle.collect_moments(g, sp, ex2, ey2, ps)
    assert got.shape == ref.shape
    assert abs(ref[0].sum() - got[0].sum()) <= 1e-5 * ref[0].sum()
    for m, name in enumerate(NAMES):
        scale = np.abs(ref[m]).max()
        assert scale > 0, name
        tol = (2e-5 if m == 0 else 2e-4) * scale
        assert np.abs(got[m] - ref[m]).max() <= tol, (name, np.abs(got[m] - ref[m]).max(), scale)
