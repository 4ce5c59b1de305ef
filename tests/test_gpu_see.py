"""Electron-induced electron emission (PROCESS_ELECTRON_INDUCED_ELECTRON_EMISSION, pic2d_SEEmission.f90:4-1208) on the
device against the oracle: electrons launched into the walls with energies from 1 to 600 eV, one electron push, and
the electrons each absorbed one produces (elastic reflection, specular or at random angles, inelastic
backscattering, true secondaries with models 1 and 2 and both yield branches), appended to the electrons at the
end of the step: identical counts per wall, rows as sets."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import ELECTRONS, PREC_FP64, PREC_MIXED, Simulation
from edipic_b200.decks import SEE_OFF
from gpu_common import oracle_geom, small_deck
from test_gpu_emission import pair_rows

# wall 0: the reference's SEE example material (all models 2, random elastic angles); wall 1: constant coefficients,
# specular elastic and a true yield above 1; walls 2, 3 (walled domain): true secondaries only / off
WALLS = {
    0: dict(SEE_OFF, elastic_model=2, elastic_type=1, elastic_e0_ev=2.0, elastic_emax_coef_ev=10.0, elastic_max=0.55,
            elastic_de_ev=14.0, elastic_frac_classic=0.03, inelastic_model=2, inelastic_frac_classic=0.07,
            true_model=2, true_t_ev=2.0, classic_e0_ev=13.0, classic_emax_ev=500.0, classic_max=3.0,
            classic_k_smooth=1.0),
    1: dict(SEE_OFF, elastic_model=1, elastic_type=0, elastic_yield=0.3, elastic_emin_ev=0.0, elastic_emax_ev=300.0,
            inelastic_model=1, inelastic_yield=0.2, inelastic_emin_ev=5.0, inelastic_emax_ev=1000.0, true_model=1,
            true_yield=1.7, true_emin_ev=8.0, true_emax_ev=400.0, true_t_ev=3.0),
    2: dict(SEE_OFF, true_model=2, true_t_ev=1.0, classic_e0_ev=20.0, classic_emax_ev=300.0, classic_max=0.8,
            classic_k_smooth=2.0),
}


def wall_electrons(sim, n, seed, precision, ef):
    p = sim.params
    rng = np.random.default_rng(seed)
    e_ev = np.exp(rng.uniform(0.0, np.log(600.0), n))
    sp = np.sqrt(e_ev / ef)
    # direction: mostly towards the wall, any angle of incidence
    ct = rng.uniform(0.05, 1.0, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    vn, t1, t2 = sp * ct, sp * np.sqrt(1 - ct ** 2) * np.cos(phi), sp * np.sqrt(1 - ct ** 2) * np.sin(phi)
    x = rng.uniform(1.0, p.ncx - 1.0, n)
    y = rng.uniform(1.0, p.ncy - 1.0, n)
    side = rng.integers(0, 2 if sim.periodic else 4, n)
    d = rng.uniform(0.0, 1.0, n) * vn          # reaches the wall within the step
    vx, vy, vz = t1.copy(), -vn, t2.copy()     # below
    hi = side == 1
    y[side == 0] = d[side == 0]
    y[hi], vy[hi] = p.ncy - 1e-4 - d[hi], vn[hi]
    for s, sign in ((2, -1.0), (3, 1.0)):      # left, right
        m = side == s
        vx[m], vy[m] = sign * vn[m], t1[m]
        x[m] = d[m] if s == 2 else p.ncx - 1e-4 - d[m]
    if precision == PREC_MIXED:
        i, j = np.floor(x), np.floor(y)
        x = i + (x - i).astype(np.float32).astype(np.float64)
        y = j + (y - j).astype(np.float32).astype(np.float64)
        vx, vy, vz = (a.astype(np.float32).astype(np.float64) for a in (vx, vy, vz))
    return x, y, vx, vy, vz


@pytest.mark.gpu
@pytest.mark.parametrize("precision,sort_every", [(PREC_MIXED, 0), (PREC_MIXED, 4), (PREC_FP64, 0)])
@pytest.mark.parametrize("geometry", ["periodic", "walled"])
def test_electron_emission_matches_oracle(tmp_path, precision, sort_every, geometry):
    kw = {"inner": False} if geometry == "walled" else {}
    d = small_deck(tmp_path, geometry, collisions=False, **kw)
    with Simulation(d, precision=precision, sort_every=sort_every, fuse_collisions=False) as sim:
        p = sim.params
        ef = sim.deck.tables.energy_factor_eV
        for w, prm in WALLS.items():
            sim.set_electron_emission(w, **prm)
        n = 12000
        x, y, vx, vy, vz = wall_electrons(sim, n, 17, precision, ef)
        ids = np.arange(n, dtype=np.uint32) * 7 + 1
        sim.upload_particles(ELECTRONS, x, y, vx, vy, vz, ids=ids)
        step = sim.counters().step
        sim.advance_electrons()
        c = sim.counters()
        emitted = sim.emission_counts()
        sim.end_ion_cycle()
        el = sim.download_particles(ELECTRONS)
    new = ~np.isin(el["id"], ids)
    got = np.stack([el[k][new] for k in ("x", "y", "vx", "vy", "vz")], axis=1)

    g = oracle_geom(sim)
    sp = pyoracle.Species(p.bx, p.by, p.bz, p.ez, 0, 0.0, p.n_subcycles, p.ions_sense_b, p.ions_sense_ez)
    ps = pyoracle.ParticleSet(x, y, vx, vy, vz, ids=ids)
    zero = np.zeros((sim.ny_ref, sim.nx_ref))
    hits, rows = pyoracle.push_hits(g, sp, zero, zero, ps)
    ems = {w: pyoracle.ElectronEmission(prm, ef) for w, prm in WALLS.items()}
    ref, per_wall = [], np.zeros(8, np.int64)
    for r in rows:
        w = int(r[0])
        if w not in ems:
            continue
        out, m = ems[w].emit(w, r[1], r[2], r[3], r[4], r[5], int(r[6]), p.seed, step, float(p.ncx), float(p.ncy))
        assert m >= 0
        per_wall[w] += m
        ref.append(out)
    ref = np.concatenate(ref) if ref else np.zeros((0, 5))
    assert np.array_equal(np.array(c.electron_hits[:8]), hits), (list(c.electron_hits[:8]), hits)
    assert np.array_equal(emitted, per_wall), (emitted, per_wall)
    assert per_wall[0] > 300 and per_wall[1] > 300
    assert got.shape == ref.shape
    vs = np.abs(ref[:, 2:]).max()
    tol = 2e-6 if precision == PREC_MIXED else 1e-12
    assert pair_rows(ref, got, np.array([1.0, 1.0, vs, vs, vs])) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_electron_emission_at_inner_objects_matches_oracle(tmp_path, precision):
    """DO_ELECTRON_COLL_WITH_INNER_OBJECT (pic2d_ElectronWallCollisions.f90:561-645) with electron-induced emission
    from a metal and a dielectric inner object (the two example materials above, keyed 4 + n): electrons launched
    into both objects from all four sides with 3 to 700 eV, one electron push without field; the electrons each object
    emits leave the side crossed first, at the crossing (PROCESS_ELECTRON_INDUCED_ELECTRON_EMISSION with the object's
    face); the dielectric's outline takes -1 per absorbed electron and +1 per emitted one. Counts per object exact,
    rows paired with the oracle's, outline charge as the dielectric tests."""
    from test_gpu_dielectric import particles_into
    from test_gpu_emission import DIEL, METAL

    from edipic_b200 import FIELD_SURFACE_CHARGE

    d = small_deck(tmp_path, "walled", ncx=64, ncy=48, inner=[METAL, DIEL], collisions=False)
    mats = {4: WALLS[0], 5: WALLS[1]}
    with Simulation(d, precision=precision, sort_every=0, fuse_collisions=False) as sim:
        p = sim.params
        ef = sim.deck.tables.energy_factor_eV
        for o, prm in mats.items():
            sim.set_electron_emission(o, **prm)
        xa = particles_into(sim, METAL, 6000, 21, 0.7, precision)
        xb = particles_into(sim, DIEL, 6000, 22, 0.7, precision)
        x, y, vx, vy, vz = (np.concatenate([a, b]) for a, b in zip(xa, xb))
        ids = np.arange(x.size, dtype=np.uint32) * 5 + 3
        sim.upload_particles(ELECTRONS, x, y, vx, vy, vz, ids=ids)
        step = sim.counters().step
        sim.advance_electrons()
        c = sim.counters()
        emitted = sim.emission_counts()
        surf_got = sim.field(FIELD_SURFACE_CHARGE)
        sim.end_ion_cycle()
        el = sim.download_particles(ELECTRONS)
    new = ~np.isin(el["id"], ids)
    got = np.stack([el[k][new] for k in ("x", "y", "vx", "vy", "vz")], axis=1)

    g = oracle_geom(sim)
    sp = pyoracle.Species(p.bx, p.by, p.bz, p.ez, 0, 0.0, p.n_subcycles, p.ions_sense_b, p.ions_sense_ez)
    ps = pyoracle.ParticleSet(x, y, vx, vy, vz, ids=ids)
    zero = np.zeros((sim.ny_ref, sim.nx_ref))
    hits, rows = pyoracle.push_hits(g, sp, zero, zero, ps)
    see = {o: pyoracle.ElectronEmission(prm, ef) for o, prm in mats.items()}
    surf = np.zeros(pyoracle.nodes_shape(g))
    ref, per_obj = [], np.zeros(8, np.int64)
    for r in rows:
        if int(r[0]) < 4:
            continue
        out = pyoracle.inner_electron_impact(g, see, {1: True}, r, p.seed, step, surf)
        per_obj[int(r[0])] += len(out)
        ref.append(out)
    ref = np.concatenate(ref) if ref else np.zeros((0, 5))
    assert np.array_equal(np.array(c.electron_hits[:8]), hits), (list(c.electron_hits[:8]), hits)
    assert hits[4] > 3000 and hits[5] > 3000
    assert np.array_equal(emitted, per_obj), (emitted, per_obj)
    assert per_obj[4] > 300 and per_obj[5] > 300
    assert got.shape == ref.shape
    vs = np.abs(ref[:, 2:]).max()
    tol = 2e-6 if precision == PREC_MIXED else 1e-12
    assert pair_rows(ref, got, np.array([1.0, 1.0, vs, vs, vs])) <= tol
    stol = 5e-4 if precision == PREC_MIXED else 1e-8
    assert np.abs(surf_got - surf).max() < stol, np.abs(surf_got - surf).max()
