"""Ion-wall interactions on the device against the oracle: ions launched into the walls, one ion push, then
* ion-induced electron emission (PROCESS_ION_INDUCED_ELECTRON_EMISSION, pic2d_IonEmissions.f90:1-348): the electrons
  emitted by each absorbed ion (count per wall, positions 1e-6 inside the wall, velocities from the injection and
  Maxwell tables scaled to the emission temperature and to the ion's energy budget), appended to the electrons at
  the end of the step;
* specular reflection (INJECT_REFLECTED_ION, :374-492) on the walls with ion-material model 1: the reflected ions
  appended to the ions at the end of the step."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import ELECTRONS, FIELD_SURFACE_CHARGE, IONS, PREC_FP64, PREC_MIXED, Simulation
from gpu_common import oracle_geom, small_deck


def wall_ions(sim, n, seed, precision):
    """Ions within one step of a wall, moving into it (bottom/top; left/right too on the walled domain)."""
    p = sim.params
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, p.ncx, n)
    y = rng.uniform(0.0, p.ncy, n)
    v = rng.normal(0.0, 0.001, (3, n))
    out = 0.0005 + np.abs(rng.normal(0.0, 0.0015, n))
    side = rng.integers(0, 2 if sim.periodic else 4, n)
    d = rng.uniform(0.0, 0.003, n)
    lo, hi = side == 0, side == 1
    y[lo], v[1][lo] = d[lo], -out[lo]
    y[hi], v[1][hi] = p.ncy - 1e-4 - d[hi], out[hi]
    if not sim.periodic:
        le, ri = side == 2, side == 3
        x[le], v[0][le] = d[le], -out[le]
        x[ri], v[0][ri] = p.ncx - 1e-4 - d[ri], out[ri]
    if precision == PREC_MIXED:
        i, j = np.floor(x), np.floor(y)
        x = i + (x - i).astype(np.float32).astype(np.float64)
        y = j + (y - j).astype(np.float32).astype(np.float64)
        v = v.astype(np.float32).astype(np.float64)
    return x, y, v[0], v[1], v[2]


def pair_rows(a, b, scale):
    """Nearest-neighbour pairing of the rows of a and b (same count, columns divided by scale); the pairing must be
    one to one. Returns the largest distance (max norm) of a pair."""
    from scipy.spatial import cKDTree

    assert a.shape == b.shape, (a.shape, b.shape)
    if a.size == 0:
        return 0.0
    d, j = cKDTree(b / scale).query(a / scale, p=np.inf)
    assert np.unique(j).size == j.size, "rows do not pair one to one"
    return float(d.max())


@pytest.mark.gpu
@pytest.mark.parametrize("precision,sort_every", [(PREC_MIXED, 0), (PREC_MIXED, 4), (PREC_FP64, 0)])
@pytest.mark.parametrize("geometry", ["periodic", "walled"])
@pytest.mark.parametrize("reflect", [False, True])
def test_ion_emission_matches_oracle(tmp_path, precision, sort_every, geometry, reflect):
    kw = {"inner": False} if geometry == "walled" else {}
    d = small_deck(tmp_path, geometry, ion_emission=False, **kw)
    with Simulation(d, precision=precision, sort_every=sort_every, fuse_collisions=False) as sim:
        p = sim.params
        ef = sim.deck.tables.energy_factor_eV
        ms = p.ion_mass_me[0]
        n = 8000
        x, y, vx, vy, vz = wall_ions(sim, n, seed=5, precision=precision)
        e_ev = ms * (vx * vx + vy * vy + vz * vz) * ef
        e0, e1 = np.percentile(e_ev, 15), np.percentile(e_ev, 85)
        walls = {w: (2.3 if w % 2 == 0 else 0.6, e0, e1, 20.0) for w in range(2 if sim.periodic else 4)}
        for w, (yld, a, b, t) in walls.items():
            sim.set_ion_emission(w, 1, yld, a, b, t)
        # with reflection: the walls below and on the left reflect (and keep their emission parameters unused)
        reflecting = {0, 2} if reflect else set()
        for w in reflecting:
            sim.set_ion_reflection(w, True)
        ne = 16
        sim.upload_particles(ELECTRONS, x[:ne], y[:ne], 0 * vx[:ne], 0 * vy[:ne], 0 * vz[:ne],
                             ids=np.arange(ne, dtype=np.uint32) + 500000)
        ids = np.arange(n, dtype=np.uint32) * 5 + 3
        sim.upload_particles(IONS, x, y, vx, vy, vz, ids=ids)
        step = sim.counters().step
        sim.advance_ions()
        emitted = sim.emission_counts()
        c = sim.counters()
        sim.end_ion_cycle()
        el = sim.download_particles(ELECTRONS)
        io = sim.download_particles(IONS)

    new = el["id"] >= 0
    new &= ~np.isin(el["id"], np.arange(ne, dtype=np.uint32) + 500000)
    got = np.stack([el[k][new] for k in ("x", "y", "vx", "vy", "vz")], axis=1)

    g = oracle_geom(sim)
    sp = pyoracle.Species(p.bx, p.by, p.bz, p.ez, 1, 0.5 * p.ion_charge[0] / p.ion_mass_me[0], p.n_subcycles,
                          p.ions_sense_b, p.ions_sense_ez)
    ps = pyoracle.ParticleSet(x, y, vx, vy, vz, ids=ids)
    zero = np.zeros((sim.ny_ref, sim.nx_ref))
    hits, rows = pyoracle.push_hits(g, sp, zero, zero, ps)
    em = pyoracle.IonEmission(walls, ms, ef)
    ref, per_wall, refl = [], np.zeros(8, np.int64), []
    for r in rows:
        if int(r[0]) in reflecting:
            refl.append(pyoracle.ion_reflect(int(r[0]), r[1], r[2], r[3], r[4], r[5], float(p.ncx), float(p.ncy)))
            continue
        out = em.emit(int(r[0]), r[1], r[2], r[3], r[4], r[5], int(r[6]), p.seed, step, float(p.ncx), float(p.ncy))
        per_wall[int(r[0])] += len(out)
        ref.append(out)
    ref = np.concatenate(ref) if ref else np.zeros((0, 5))

    assert np.array_equal(np.array(c.ion_hits[:8]), hits), (list(c.ion_hits[:8]), hits)
    # reflected ions: the ions that are not original
    back = ~np.isin(io["id"], ids)
    got_i = np.stack([io[k][back] for k in ("x", "y", "vx", "vy", "vz")], axis=1)
    ref_i = np.array(refl).reshape(-1, 5)
    assert (len(ref_i) > 300) == reflect
    assert got_i.shape == ref_i.shape
    if reflect:
        vs = np.abs(ref_i[:, 2:]).max()
        assert pair_rows(ref_i, got_i, np.array([1.0, 1.0, vs, vs, vs])) <= (2e-6 if precision == PREC_MIXED else 1e-12)
    assert np.array_equal(emitted, per_wall), (emitted, per_wall)
    assert per_wall.sum() > 500
    assert got.shape == ref.shape
    vscale = np.abs(ref[:, 2:]).max()
    scale = np.array([1.0, 1.0, vscale, vscale, vscale])
    tol = 2e-6 if precision == PREC_MIXED else 1e-12
    assert pair_rows(ref, got, scale) <= tol
    # the electrons start 1e-6 inside the wall they came from
    on_wall = (np.abs(ref[:, 1] - 1e-6) < 1e-9) | (np.abs(ref[:, 1] - (p.ncy - 1e-6)) < 1e-9)
    if not sim.periodic:
        on_wall |= (np.abs(ref[:, 0] - 1e-6) < 1e-9) | (np.abs(ref[:, 0] - (p.ncx - 1e-6)) < 1e-9)
    assert on_wall.all()


METAL = (20, 24, 36, 32, -100.0)
DIEL = (44, 10, 54, 20, 0.0, 4.0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
@pytest.mark.parametrize("reflect", [False, True])
def test_ion_impacts_on_inner_objects_match_oracle(tmp_path, precision, reflect):
    """DO_ION_COLL_WITH_INNER_OBJECT (pic2d_IonWallCollisions.f90:484-575) for ions launched into a metal and a
    dielectric inner object from all four sides, one ion push without field: the electrons each object emits leave
    the side the ion crossed first, 1e-6 outside it at the crossing point (INJECT_ION_IMPACT_EXTRACTED_ELECTRON with
    m = -1, pic2d_IonEmissions.f90:232-330); the dielectric's outline takes the ion's charge and +1 per emitted
    electron; with reflection the metal object returns its ions instead (INJECT_REFLECTED_ION, :430-470). Counts per
    object are exact; rows pair with the oracle's to 2e-6 (mixed: FP32 positions) or 1e-12; outline charge as the
    dielectric tests."""
    from test_gpu_dielectric import particles_into

    d = small_deck(tmp_path, "walled", ncx=64, ncy=48, inner=[METAL, DIEL], collisions=False, ion_emission=False)
    with Simulation(d, precision=precision, sort_every=0, fuse_collisions=False) as sim:
        p = sim.params
        ef = sim.deck.tables.energy_factor_eV
        ms = p.ion_mass_me[0]
        xa = particles_into(sim, METAL, 6000, 11, 0.3, precision)
        xb = particles_into(sim, DIEL, 6000, 12, 0.3, precision)
        x, y, vx, vy, vz = (np.concatenate([a, b]) for a, b in zip(xa, xb))
        e_ev = ms * (vx * vx + vy * vy + vz * vz) * ef
        e0, e1 = np.percentile(e_ev, 10), np.percentile(e_ev, 90)
        objs = {4: (1.7, e0, e1, 15.0), 5: (0.8, e0, e1, 5.0)}
        for o, (yld, a, b, t) in objs.items():
            sim.set_ion_emission(o, 1, yld, a, b, t)
        if reflect:
            sim.set_ion_reflection(4, True)
        n = x.size
        ids = np.arange(n, dtype=np.uint32) * 3 + 7
        sim.upload_particles(ELECTRONS, x[:8], y[:8], 0 * x[:8], 0 * x[:8], 0 * x[:8],
                             ids=np.arange(8, dtype=np.uint32) + 900000)
        sim.upload_particles(IONS, x, y, vx, vy, vz, ids=ids)
        step = sim.counters().step
        sim.advance_ions()
        emitted = sim.emission_counts()
        c = sim.counters()
        surf_got = sim.field(FIELD_SURFACE_CHARGE)
        sim.end_ion_cycle()
        el = sim.download_particles(ELECTRONS)
        io = sim.download_particles(IONS)

    g = oracle_geom(sim)
    sp = pyoracle.Species(p.bx, p.by, p.bz, p.ez, 1, 0.5 * p.ion_charge[0] / p.ion_mass_me[0], p.n_subcycles,
                          p.ions_sense_b, p.ions_sense_ez)
    ps = pyoracle.ParticleSet(x, y, vx, vy, vz, ids=ids)
    zero = np.zeros((sim.ny_ref, sim.nx_ref))
    hits, rows = pyoracle.push_hits(g, sp, zero, zero, ps)
    em = pyoracle.IonEmission(objs, ms, ef)
    surf = np.zeros(pyoracle.nodes_shape(g))
    ref, refl, per_obj = [], [], np.zeros(8, np.int64)
    for r in rows:
        if int(r[0]) < 4:
            continue
        out, back = pyoracle.inner_ion_impact(g, em, {4: reflect}, {1: True}, float(p.ion_charge[0]), r, p.seed,
                                              step, float(p.n_subcycles), surf)
        if back is not None:
            refl.append(back)
        per_obj[int(r[0])] += len(out)
        ref.append(out)
    ref = np.concatenate(ref)
    assert np.array_equal(np.array(c.ion_hits[:8]), hits) and hits[4] > 1000 and hits[5] > 1000
    assert np.array_equal(emitted, per_obj), (emitted, per_obj)
    assert per_obj[5] > 300 and (per_obj[4] == 0) == reflect
    new = ~np.isin(el["id"], np.arange(8, dtype=np.uint32) + 900000)
    got = np.stack([el[k][new] for k in ("x", "y", "vx", "vy", "vz")], axis=1)
    tol = 2e-6 if precision == PREC_MIXED else 1e-12
    vs = np.abs(ref[:, 2:]).max()
    assert pair_rows(ref, got, np.array([1.0, 1.0, vs, vs, vs])) <= tol
    back = ~np.isin(io["id"], ids)
    got_i = np.stack([io[k][back] for k in ("x", "y", "vx", "vy", "vz")], axis=1)
    ref_i = np.array(refl).reshape(-1, 5)
    assert got_i.shape == ref_i.shape and (len(ref_i) > 1000) == reflect
    if reflect:
        vs = np.abs(ref_i[:, 2:]).max()
        assert pair_rows(ref_i, got_i, np.array([1.0, 1.0, vs, vs, vs])) <= tol
    stol = 5e-4 if precision == PREC_MIXED else 1e-8
    assert np.abs(surf_got - surf).max() < stol, np.abs(surf_got - surf).max()
