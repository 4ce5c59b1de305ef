"""Field solves on the device against the oracle on the same charge density: FFT_X (SOLVE_POISSON_FFTX_LINSYSY)
to 1e-9 of max|phi|, E from phi, and the CG replacement of the PETSc solve to the discrete operator's solution."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import (ELECTRONS, FIELD_EX, FIELD_EY, FIELD_PHI, FIELD_RHO_TOTAL, IONS, PREC_FP64, PREC_MIXED,
                         PRECOND_MG, PRECOND_NONE, Simulation, WARM_ZERO)
from gpu_common import oracle_geom, random_particles, small_deck


def _load_plasma(sim, precision, seed=4):
    n = sim.params.ncx * sim.params.ncy * 12
    xe = random_particles(sim, n, seed=seed, precision=precision)
    xi = random_particles(sim, n // 2, seed=seed + 1, precision=precision, vscale=0.001)
    sim.upload_particles(ELECTRONS, *xe)
    sim.upload_particles(IONS, *xi)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
@pytest.mark.parametrize("ncx,ncy", [(64, 48), (256, 40)])
def test_fftx_matches_oracle(tmp_path, precision, ncx, ncy):
    d = small_deck(tmp_path, "periodic", ncx=ncx, ncy=ncy, wall_potentials={2: 30.0, 4: -10.0})
    with Simulation(d, precision=precision, sort_every=0) as sim:
        _load_plasma(sim, precision)
        p = sim.params
        phi = sim.solve_poisson_fftx_linsysy(want_phi=True)
        rho_e = sim.gather_electron_charge_density()
        rho_i = sim.gather_ion_charge_density()
        rho_t = sim.field(FIELD_RHO_TOTAL)
        ex, ey = sim.field(FIELD_EX), sim.field(FIELD_EY)
    g = oracle_geom(sim)
    rho = (rho_i - rho_e) / p.n_of_particles_cell
    assert np.allclose(rho_t, rho, rtol=0, atol=1e-12 * max(1.0, np.abs(rho).max()))
    ref = pyoracle.fftx_solve(g, rho, p.wall_phi_const[0], p.wall_phi_const[1])
    assert np.abs(phi - ref).max() <= 1e-9 * np.abs(ref).max()
    f2 = p.f_scale_v / (p.e_scale_vm * 2.0 * p.delta_x_m)
    f1 = p.f_scale_v / (p.e_scale_vm * p.delta_x_m)
    rex, rey = pyoracle.efield(g, phi, f2, f1)
    tol = (1e-6 if precision == PREC_MIXED else 1e-12) * max(np.abs(rex).max(), np.abs(rey).max())
    assert np.abs(ex - rex).max() <= tol and np.abs(ey - rey).max() <= tol
    # the discrete operator of the reference: phi_{j-1} + phi_{j+1} + (spectral x) = -rho inside
    assert abs(phi[0, 5] - p.wall_phi_const[0]) < 1e-9 and abs(phi[-1, 5] - p.wall_phi_const[1]) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("precision,precond", [(PREC_MIXED, PRECOND_MG), (PREC_FP64, PRECOND_MG),
                                               (PREC_FP64, PRECOND_NONE)])
def test_cg_matches_oracle(tmp_path, precision, precond):
    d = small_deck(tmp_path, "walled", ncx=96, ncy=80, inner=(30, 20, 60, 36, -100.0))
    with Simulation(d, precision=precision, sort_every=0) as sim:
        sim.set_cg_preconditioner(precond)
        _load_plasma(sim, precision)
        p = sim.params
        it = sim.solve_potential_with_cg(rtol=1e-12, max_it=20000, warm_start=WARM_ZERO)
        phi = sim.field(FIELD_PHI)
        rho_t = sim.field(FIELD_RHO_TOTAL)
        ex = sim.field(FIELD_EX)
        it2 = sim.solve_potential_with_cg(rtol=1e-8, max_it=20000)   # warm start from the converged phi
    g = oracle_geom(sim)
    ref, it_ref, rel = pyoracle.cg_solve(g, rho_t, [0.0, 0.0, 0.0, 0.0], [p.inner_phi[0]], rtol=1e-13)
    assert it_ref > 0 and rel < 1e-13
    assert np.abs(phi - ref).max() <= 1e-8 * np.abs(ref).max()
    assert it > (3 if precond == PRECOND_MG else 10) and it2 <= 2
    assert np.allclose(phi[20:37, 30:61], p.inner_phi[0])
    f2 = p.f_scale_v / (p.e_scale_vm * 2.0 * p.delta_x_m)
    f1 = p.f_scale_v / (p.e_scale_vm * p.delta_x_m)
    rex, _ = pyoracle.efield(g, phi, f2, f1)
    assert np.abs(ex - rex).max() <= (1e-6 if precision == PREC_MIXED else 1e-12) * np.abs(rex).max()


@pytest.mark.gpu
@pytest.mark.parametrize("ncx,ncy,inner", [(256, 256, (96, 48, 160, 80, -100.0)), (90, 70, (20, 20, 41, 33, -50.0)),
                                           (128, 64, (30, 10, 61, 25, -200.0))])
def test_multigrid_pcg(tmp_path, ncx, ncy, inner):
    """The multigrid-preconditioned CG reaches the oracle's solution of the same operator in far fewer iterations
    than plain CG, on grids whose sizes halve many times, once (90 x 70) and with an object off the coarse
    nodes."""
    d = small_deck(tmp_path, "walled", ncx=ncx, ncy=ncy, inner=inner)
    its = {}
    with Simulation(d, precision=PREC_FP64, sort_every=0) as sim:
        _load_plasma(sim, PREC_FP64)
        p = sim.params
        for pc in (PRECOND_NONE, PRECOND_MG):
            sim.set_cg_preconditioner(pc)
            its[pc] = sim.solve_potential_with_cg(rtol=1e-10, max_it=50000, warm_start=WARM_ZERO)
            phi = sim.field(FIELD_PHI)
            rho_t = sim.field(FIELD_RHO_TOTAL)
            c = sim.counters()
            assert c.cg_relres <= 1e-10 and c.cg_iterations == its[pc]
            g = oracle_geom(sim)
            ref, _, _ = pyoracle.cg_solve(g, rho_t, [0.0] * 4, [p.inner_phi[0]], rtol=1e-13)
            assert np.abs(phi - ref).max() <= 1e-8 * np.abs(ref).max()
    assert its[PRECOND_MG] * 4 < its[PRECOND_NONE]
    if ncx == 256:
        assert its[PRECOND_MG] <= 20


@pytest.mark.gpu
def test_time_dependent_potentials_reach_the_field_solve(tmp_path):
    """UPDATE_WALL_POTENTIALS with a pulsed custom waveform on the top wall (FFT_X) and a harmonically oscillating
    metal inner object (CG): after edp_update_wall_potentials(T) for consecutive T, the solved potential on the wall
    row and on the object's nodes equals the oracle's restatement of the potential at T."""
    d = small_deck(tmp_path / "p", "periodic", ncx=64, ncy=48, wall_potentials={2: 12.0},
                   oscillations={2: (30.0, 731.0, 15.0)},
                   waveforms={2: (50.0, 1.0e9, [(0.0, -1.0), (0.49, -0.5), (0.51, 1.0), (1.0, 0.5)])},
                   amplitude_profiles={2: [(0.0, 1.0), (5.0, 1.0), (5.0, 0.0), (19.5, 0.0)]})
    prof = pyoracle.wall_profiles(d)
    with Simulation(d, sort_every=0) as sim:
        _load_plasma(sim, PREC_MIXED)
        checked = 0
        for t in range(0, 4200):
            sim.update_wall_potentials(t)
            want = prof[1].value(t)
            prof[0].value(t)
            if t % 97 == 0 or t in (998, 999, 1000, 1001, 3799, 3800, 3801):
                phi = sim.solve_poisson_fftx_linsysy(want_phi=True)
                assert abs(phi[-1, 7] - want) <= 1e-12 * max(1.0, abs(want)), t
                checked += 1
        assert checked > 40
    dw = small_deck(tmp_path / "w", "walled", ncx=64, ncy=64, inner=(20, 24, 36, 32, -40.0),
                    oscillations={5: (25.0, 1000.0, 45.0)})
    prof = pyoracle.wall_profiles(dw)
    with Simulation(dw, sort_every=0) as sim:
        _load_plasma(sim, PREC_MIXED)
        for t in range(0, 60):
            sim.update_wall_potentials(t)
            want = prof[4].value(t)
            if t % 7 == 0:
                sim.solve_potential_with_cg(rtol=1e-10, max_it=5000)
                phi = sim.field(FIELD_PHI)
                assert np.abs(phi[24:33, 20:37] - want).max() <= 1e-12 * max(1.0, abs(want)), t
