"""Dielectric inner objects on the device against the oracle:
* the CG solve with the face permittivities of SET_EPS_ISHIFTED/JSHIFTED (pic2d_PETSc_Solver.F90:1724-2045), a metal
  and a dielectric object, with and without the multigrid preconditioner, and the outline's surface charge entering
  the density (pic2d_ElectronDynamics.f90:1903-1909);
* electrons and ions absorbed by the dielectric putting their charge on the outline nodes next to the crossing of
  their trajectory (DO_ELECTRON_COLL_WITH_INNER_OBJECT / DO_ION_COLL_WITH_INNER_OBJECT)."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import (ELECTRONS, FIELD_PHI, FIELD_RHO_TOTAL, FIELD_SURFACE_CHARGE, IONS, PREC_FP64, PREC_MIXED,
                         PRECOND_MG, PRECOND_NONE, Simulation, WARM_ZERO)
from gpu_common import oracle_geom, random_particles, small_deck

METAL = (20, 24, 36, 32, -100.0)
DIEL = (44, 10, 54, 20, 0.0, 4.0)


@pytest.mark.gpu
@pytest.mark.parametrize("precond", [PRECOND_MG, PRECOND_NONE])
def test_dielectric_cg_matches_oracle(tmp_path, precond):
    d = small_deck(tmp_path, "walled", ncx=64, ncy=48, inner=[METAL, DIEL], collisions=False)
    with Simulation(d, precision=PREC_FP64, sort_every=0) as sim:
        p = sim.params
        assert list(p.inner_eps)[:2] == [0.0, 4.0]
        sim.set_cg_preconditioner(precond)
        n = p.ncx * p.ncy * 12
        sim.upload_particles(ELECTRONS, *random_particles(sim, n, seed=2, precision=PREC_FP64))
        sim.upload_particles(IONS, *random_particles(sim, n // 2, seed=3, precision=PREC_FP64, vscale=0.001))
        sim.solve_potential_with_cg(rtol=1e-12, max_it=20000, warm_start=WARM_ZERO)
        rho0 = sim.field(FIELD_RHO_TOTAL)
        surf = np.zeros_like(rho0)
        il, jb, ir, jt = DIEL[:4]
        rng = np.random.default_rng(5)
        for i in range(il, ir + 1):
            surf[jb, i], surf[jt, i] = rng.normal(0, 30), rng.normal(0, 30)
        for j in range(jb, jt + 1):
            surf[j, il], surf[j, ir] = rng.normal(0, 30), rng.normal(0, 30)
        sim.set_field(FIELD_SURFACE_CHARGE, surf)
        it = sim.solve_potential_with_cg(rtol=1e-12, max_it=20000, warm_start=WARM_ZERO)
        rho1 = sim.field(FIELD_RHO_TOTAL)
        phi = sim.field(FIELD_PHI)
        back = sim.field(FIELD_SURFACE_CHARGE)
    assert np.abs(back - surf).max() < 1e-9
    assert np.abs((rho1 - rho0) - surf / p.n_of_particles_cell).max() < 1e-9
    g = oracle_geom(sim)
    ref, it_ref, rel = pyoracle.cg_solve_eps(g, rho1, [0.0] * 4, [p.inner_phi[0], 0.0], [0.0, 4.0], rtol=1e-13)
    assert rel < 1e-13 and it > 3
    assert np.abs(phi - ref).max() <= 1e-8 * np.abs(ref).max()
    assert np.allclose(phi[METAL[1]:METAL[3] + 1, METAL[0]:METAL[2] + 1], p.inner_phi[0])


def particles_into(sim, obj, n, seed, vmax, precision):
    """Particles within one step of the object's sides, moving into it."""
    il, jb, ir, jt = obj[:4]
    rng = np.random.default_rng(seed)
    side = rng.integers(0, 4, n)
    s = rng.uniform(0.0, 1.0, n)
    vn = rng.uniform(0.05, vmax, n)
    vt = rng.uniform(-0.5, 0.5, n) * vmax
    d = rng.uniform(0.0, 1.0, n) * vn
    x = np.where(side < 2, il + s * (ir - il), 0.0)
    y = np.where(side >= 2, jb + s * (jt - jb), 0.0)
    vx, vy = vt.copy(), vt.copy()
    m = side == 0   # below the bottom side, moving up
    y[m], vy[m] = jb - d[m], vn[m]
    m = side == 1   # above the top side
    y[m], vy[m] = jt + d[m], -vn[m]
    m = side == 2   # left of the left side
    x[m], vx[m] = il - d[m], vn[m]
    m = side == 3
    x[m], vx[m] = ir + d[m], -vn[m]
    vz = rng.normal(0, 0.01, n)
    if precision == PREC_MIXED:
        i, j = np.floor(x), np.floor(y)
        x = i + (x - i).astype(np.float32).astype(np.float64)
        y = j + (y - j).astype(np.float32).astype(np.float64)
        vx, vy, vz = (a.astype(np.float32).astype(np.float64) for a in (vx, vy, vz))
    return x, y, vx, vy, vz


@pytest.mark.gpu
@pytest.mark.parametrize("precision,sort_every", [(PREC_MIXED, 0), (PREC_MIXED, 4), (PREC_FP64, 0)])
def test_outline_charge_matches_oracle(tmp_path, precision, sort_every):
    d = small_deck(tmp_path, "walled", ncx=64, ncy=48, inner=[METAL, DIEL], collisions=False)
    with Simulation(d, precision=precision, sort_every=sort_every, fuse_collisions=False) as sim:
        p = sim.params
        xe = particles_into(sim, DIEL, 20000, 7, 0.6, precision)
        xi = particles_into(sim, DIEL, 10000, 8, 0.3, precision)
        sim.upload_particles(ELECTRONS, *xe)
        sim.upload_particles(IONS, *xi)
        sim.advance_electrons()   # no field: straight moves
        sim.advance_ions()
        c = sim.counters()
        got = sim.field(FIELD_SURFACE_CHARGE)
    g = oracle_geom(sim)
    surf = np.zeros(pyoracle.nodes_shape(g))
    il, jb, ir, jt = DIEL[:4]
    hits = 0
    for (x, y, vx, vy, _), q, xmul in ((xe, -1.0, 1.0), (xi, float(p.ion_charge[0]), float(p.n_subcycles))):
        X, Y = x + vx * xmul, y + vy * xmul
        inside = (X > il) & (X < ir) & (Y > jb) & (Y < jt)
        hits += inside.sum()
        for k in np.nonzero(inside)[0]:
            assert pyoracle.inner_hit(g, [0.0, 4.0], X[k], Y[k], vx[k], vy[k], xmul, q, surf) == 1
    assert hits > 10000
    assert c.electron_hits[5] + c.ion_hits[5] == hits
    tol = 5e-4 if precision == PREC_MIXED else 1e-8
    assert np.abs(got - surf).max() < tol, np.abs(got - surf).max()
    assert abs(got.sum() - surf.sum()) < tol * 10
