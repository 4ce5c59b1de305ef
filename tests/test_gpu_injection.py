"""Constant electron emission of the walls (PERFORM_ELECTRON_EMISSION_SETUP, pic2d_Setup.f90:599-1001) on the device
against the oracle over three steps: counts per wall (integer part plus the Bernoulli fraction), places along the
walls, thermal and beam normal speeds and Maxwellian tangential components, appended to the electrons at the end of
each step; the deck's init_bo_NN.dat values reach the context."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import ELECTRONS, PREC_FP64, PREC_MIXED, Simulation
from gpu_common import oracle_geom, small_deck
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
        # N_electron_constant_emit is a REAL: the deck keeps it in single precision
        assert sim.deck.wall_injection == {w: (float(np.float32(a)), b, float(c), float(e), float(f))
                                           for w, (a, b, c, e, f) in inj.items()}
        inj = dict(sim.deck.wall_injection)
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


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_inner_object_injection_matches_oracle(tmp_path, precision):
    """PERFORM_ELECTRON_EMISSION_SETUP_INNER_OBJECTS (pic2d_Setup.f90:1005-1591) for three metal inner objects of a
    walled domain: one free, one attached to its right side (each covers part of the other's side), one standing on
    the bottom wall (its bottom side covered): counts per side in single precision REAL(N) REAL(open) / REAL(L),
    places by the walk over the open cells, 1e-6 outside, normal velocities out; from the deck's init_bo_NN.dat."""
    inner = [(20, 24, 36, 32, -100.0), (36, 26, 44, 30, -100.0), (50, 0, 56, 10, 0.0)]
    inj = {4: (33.3, 0, 2.0, 1.0, 0.0), 5: (6.1, 1, 1.5, 0.5, 30.0), 6: (12.7, 0, 0.5, 3.0, 0.0)}
    d = small_deck(tmp_path, "walled", ncx=64, ncy=48, inner=inner, collisions=False, wall_injection=inj)
    with Simulation(d, precision=precision, sort_every=0, fuse_collisions=False) as sim:
        assert sorted(sim.deck.wall_injection) == [4, 5, 6]
        p = sim.params
        ef = sim.deck.tables.energy_factor_eV
        sim.upload_particles(ELECTRONS, np.array([10.5]), np.array([40.5]), np.zeros(1), np.zeros(1), np.zeros(1),
                             ids=np.array([4000000000], dtype=np.uint32))
        steps = []
        for _ in range(2):
            steps.append(int(sim.counters().step))
            sim.end_ion_cycle()   # no push: every injected electron stays where it was placed
        got_counts = sim.emission_counts()
        el = sim.download_particles(ELECTRONS)
    g = oracle_geom(sim)
    ref, counts = [], np.zeros(8, np.int64)
    for t in steps:
        for obj, v in inj.items():
            rows, per = pyoracle.inner_injection(g, obj - 4, *v, ef, t, p.seed)
            counts[obj] += per.sum()
            ref.append(rows)
    ref = np.concatenate(ref)
    assert np.array_equal(got_counts, counts), (got_counts, counts)
    # the free object's sides all emit; the others have covered cells: the object on the wall emits nothing below
    r0, per0 = pyoracle.inner_injection(g, 2, *inj[6], ef, steps[0], p.seed)
    assert per0[3] == 0 and per0[0] > 0
    new = el["id"] != 4000000000
    got = np.stack([el[k][new] for k in ("x", "y", "vx", "vy", "vz")], axis=1)
    assert got.shape == ref.shape and len(ref) > 80
    vs = np.abs(ref[:, 2:]).max()
    tol = 2e-6 if precision == PREC_MIXED else 1e-12
    assert pair_rows(ref, got, np.array([1.0, 1.0, vs, vs, vs])) <= tol
