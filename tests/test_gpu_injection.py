"""Constant electron emission of the walls (PERFORM_ELECTRON_EMISSION_SETUP, pic2d_Setup.f90:599-1001) on the device
against the oracle over three steps: counts per wall (integer part plus the Bernoulli fraction), places along the
walls, thermal and beam normal speeds and Maxwellian tangential components, appended to the electrons at the end of
each step; the deck's init_bo_NN.dat values reach the context."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import ELECTRONS, PREC_FP64, PREC_MIXED, Simulation
from gpu_common import small_deck
from test_gpu_emission import pair_rows

INJ = {0: (40.3, 1, 1.5, 0.5, 60.0), 1: (25.0, 0, 2.0, 1.0, 0.0), 2: (7.7, 0, 0.5, 3.0, 0.0), 3: (0.4, 1, 2.0, 2.0, 9.0)}


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
@pytest.mark.parametrize("geometry", ["periodic", "walled"])
def test_wall_injection_matches_oracle(tmp_path, precision, geometry):
    periodic = geometry == "periodic"
    inj = {w: v for w, v in INJ.items() if not (periodic and w >= 2)}
    kw = {} if periodic else {"inner": False}
    d = small_deck(tmp_path, geometry, collisions=False, wall_injection=inj, **kw)
    with Simulation(d, precision=precision, sort_every=0, fuse_collisions=False) as sim:
        assert sim.deck.wall_injection == {w: (float(a), b, float(c), float(e), float(f))
                                           for w, (a, b, c, e, f) in inj.items()}
        p = sim.params
        ef = sim.deck.tables.energy_factor_eV
        sim.upload_particles(ELECTRONS, np.array([10.5]), np.array([10.5]), np.zeros(1), np.zeros(1), np.zeros(1))
        steps = []
        for _ in range(3):
            steps.append(int(sim.counters().step))
            sim.advance_electrons()   # the injected electrons of the previous step move once before the next ones
            sim.end_ion_cycle()
        got_counts = sim.emission_counts()
        # one more push-free view of the last step's electrons: those born at the end of the last step
        el = sim.download_particles(ELECTRONS)
    ref = [pyoracle.wall_injection(w, *v, ef, steps[-1], p.seed, float(p.ncx), float(p.ncy)) for w, v in inj.items()]
    counts = np.zeros(8, np.int64)
    for t in steps:
        for w, v in inj.items():
            counts[w] += len(pyoracle.wall_injection(w, *v, ef, t, p.seed, float(p.ncx), float(p.ncy)))
    assert np.array_equal(got_counts, counts), (got_counts, counts)
    ref = np.concatenate(ref)
    # the last step's electrons have not been pushed: find them among all electrons
    rows = np.stack([el[k] for k in ("x", "y", "vx", "vy", "vz")], axis=1)
    last = rows[-len(ref):]
    vs = np.abs(ref[:, 2:]).max()
    tol = 2e-6 if precision == PREC_MIXED else 1e-12
    assert pair_rows(ref, last, np.array([1.0, 1.0, vs, vs, vs])) <= tol
    assert np.all(ref[:, 2:][ref[:, 1] == 1e-6][:, 1] >= 0)   # below: moving up
