"""CALCULATE_ELECTRON_VDF / CALCULATE_ION_VDF (pic2d_VelocityDistributions.f90:3-393) on the device against the oracle
on the same particles, bit for bit: the 1D histograms of vx, vy, vz per box, the 2D vx-vy histogram and the count of
particles outside the bins; sorted and unsorted mixed-precision layouts with dead slots, and the FP64 path. The
large-bin case exercises the global-memory histogram path."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import ELECTRONS, FIELD_ACC_EX, FIELD_ACC_EY, FIELD_EX, FIELD_EY, IONS, PREC_FP64, PREC_MIXED, Simulation
from gpu_common import random_field, random_particles, small_deck

CASES = [((1, 1), 4, 10, True), ((3, 2), 3, 8, True), ((9, 9), 200, 100, False)]


@pytest.mark.gpu
@pytest.mark.parametrize("precision,sort_every", [(PREC_MIXED, 4), (PREC_MIXED, 0), (PREC_FP64, 0)])
@pytest.mark.parametrize("geometry", ["periodic", "walled"])
@pytest.mark.parametrize("species", [ELECTRONS, IONS])
def test_vdf_matches_oracle(tmp_path, precision, sort_every, geometry, species):
    d = small_deck(tmp_path, geometry)
    with Simulation(d, precision=precision, sort_every=sort_every, fuse_collisions=False) as sim:
        p = sim.params
        n = 50000
        x, y, vx, vy, vz = random_particles(sim, n, seed=41 + species, precision=precision,
                                            vscale=0.05 if species == ELECTRONS else 0.0003)
        sim.upload_particles(ELECTRONS, x, y, vx, vy, vz)
        if species == IONS:
            sim.upload_particles(IONS, x, y, vx, vy, vz)
        ex, ey = random_field(sim, precision=precision, amp=0.02)
        sim.set_field(FIELD_EX, ex)
        sim.set_field(FIELD_EY, ey)
        sim.set_field(FIELD_ACC_EX, ex)
        sim.set_field(FIELD_ACC_EY, ey)
        sim.advance_electrons()   # absorbed particles leave dead slots
        if species == IONS:
            sim.advance_ions()
        got = [sim.calculate_vdf(species, nbox, nmv, nvb, two_d) for nbox, nmv, nvb, two_d in CASES]
        parts = sim.download_particles(species)
        nmv_scale = sim.deck.n_max_vel
    ps = pyoracle.ParticleSet(parts["x"], parts["y"], parts["vx"], parts["vy"], parts["vz"])
    for (nbox, nmv, nvb, two_d), (h1, h2, sk) in zip(CASES, got):
        fvc = float(nmv_scale * nvb) * (np.sqrt(p.ion_mass_me[0]) if species == IONS else 1.0)
        xarea = float(p.ncx + 1 if sim.periodic else p.ncx)   # c_X_area_max of the one cluster
        r1, r2, rs = pyoracle.vdf(ps, nbox, xarea, float(p.ncy), fvc, nmv, nvb, two_d)
        assert np.array_equal(h1, r1), (nbox, np.abs(h1 - r1).max())
        assert sk == rs
        assert h1[0].sum() + sk == parts["x"].size
        if two_d:
            assert np.array_equal(h2, r2)
            assert np.array_equal(h2.sum(axis=1), h1[0])
    assert got[0][2] > 0 and got[1][2] > got[0][2]   # fast particles fall outside the narrower bins
