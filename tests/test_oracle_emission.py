"""The oracle's ion-induced electron emission (oracle_ion_emission, restating pic2d_IonEmissions.f90:1-348) against
the properties the reference's algorithm fixes: the mean number of electrons per ion equals the yield inside the
energy window and is zero outside it, every electron starts 1e-6 inside its wall and moves away from it, the normal
speed follows the flux-weighted half-Maxwellian of GetInjMaxwellVelocity (mean sqrt(pi)/2 in thermal units) and the
tangential components the Maxwellian of GetMaxwellVelocity (mean square 1/2), and the electrons never carry more than
the ion's energy above E_min."""
import numpy as np

import pyoracle

EF = 1000.0       # energy_factor_eV of the test units
MS = 72915.0      # Ar+ mass in electron masses
XMAX, YMAX = 64.0, 48.0


def emitter(yld, e0=10.0, e1=5000.0, t=2.0, walls=(0, 1, 2, 3)):
    return pyoracle.IonEmission({w: (yld, e0, e1, t) for w in walls}, MS, EF)


def ion_speed(e_ev):
    return np.sqrt(e_ev / EF / MS)


def test_mean_yield_and_window():
    em = emitter(2.3)
    v = ion_speed(1000.0)
    counts = [len(em.emit(0, 10.0, -0.01, 0.0, -v, 0.0, k, 7, 3, XMAX, YMAX)) for k in range(20000)]
    counts = np.array(counts)
    assert set(np.unique(counts)) == {2, 3}
    assert abs(counts.mean() - 2.3) < 4 * np.sqrt(0.3 * 0.7 / counts.size)
    # outside (E_min, E_max): nothing
    assert len(em.emit(0, 10.0, -0.01, 0.0, -ion_speed(5.0), 0.0, 1, 7, 3, XMAX, YMAX)) == 0
    assert len(em.emit(0, 10.0, -0.01, 0.0, -ion_speed(6000.0), 0.0, 1, 7, 3, XMAX, YMAX)) == 0
    # a wall without emission
    assert len(emitter(2.3, walls=(1,)).emit(0, 10.0, -0.01, 0.0, -v, 0.0, 1, 7, 3, XMAX, YMAX)) == 0


def test_positions_directions_and_distributions():
    t_emit = 2.0
    f = np.sqrt(t_emit / EF)
    em = emitter(1.0, t=t_emit)
    v = ion_speed(2000.0)
    cases = {0: (10.0, -0.01, 0.0, -v, 1, 1e-6), 1: (10.0, YMAX + 0.01, 0.0, v, 1, YMAX - 1e-6),
             2: (-0.01, 20.0, -v, 0.0, 0, 1e-6), 3: (XMAX + 0.01, 20.0, v, 0.0, 0, XMAX - 1e-6)}
    for wall, (x, y, vx, vy, axis, pos) in cases.items():
        rows = np.concatenate([em.emit(wall, x, y, vx, vy, 0.0, k, 11, 5, XMAX, YMAX) for k in range(30000)])
        assert rows.shape == (30000, 5)
        assert np.all(rows[:, axis] == pos)
        other = 1 - axis
        assert np.all(rows[:, other] == (10.0 if axis == 1 else 20.0))
        sign = 1.0 if wall in (0, 2) else -1.0
        normal = sign * rows[:, 2 + axis] / f
        assert np.all(normal >= 0.0)
        assert abs(normal.mean() - np.sqrt(np.pi) / 2) < 0.01
        tang = rows[:, [2 + other, 4]] / f
        assert abs((tang ** 2).mean() - 0.5) < 0.01
        assert abs(tang.mean()) < 0.01


def test_energy_budget():
    # a hot emission temperature: most ions cannot pay for three electrons
    em = emitter(3.0, e0=10.0, t=50.0)
    for k in range(3000):
        e_ion = 10.0 + 200.0 * ((k * 0.618034) % 1.0) + 1e-3
        rows = em.emit(0, 5.0, -0.01, 0.0, -ion_speed(e_ion), 0.0, k, 13, 9, XMAX, YMAX)
        spent = (rows[:, 2:] ** 2).sum() * EF
        assert spent <= (e_ion - 10.0) * (1 + 1e-9)
        assert 1 <= len(rows) <= 3


def test_inner_injection_places_electrons_on_open_cells():
    """oracle_inner_injection (PERFORM_ELECTRON_EMISSION_SETUP_INNER_OBJECTS, pic2d_Setup.f90:1005-1591): an object
    on the bottom wall emits nothing below; where another object covers part of a side, no electron starts there; the
    per-side counts follow REAL(N) REAL(open) / REAL(L); every electron starts 1e-6 outside a side and moves out."""
    g = pyoracle.geom(64, 48, False, [(20, 24, 36, 32), (36, 26, 44, 30), (50, 0, 56, 10)])
    tot = np.zeros(4)
    steps = 400
    for t in range(steps):
        rows, per = pyoracle.inner_injection(g, 0, 10.0, 0, 2.0, 1.0, 0.0, EF, t, 77)
        tot += per
        right = rows[np.isclose(rows[:, 0], 36 + 1e-6, atol=1e-9)]
        # object 1 covers the cells 26..29 of object 0's right side
        assert np.all((right[:, 1] < 26) | (right[:, 1] >= 30)) and np.all(right[:, 2] > 0)
        left = rows[np.isclose(rows[:, 0], 20 - 1e-6, atol=1e-9)]
        assert np.all(left[:, 2] < 0)
    # L = 8 + 16 + 4 + 16 = 44 open cells (right side 8 - 4 covered): rates 8, 16, 4, 16 of 44 per 10 electrons
    np.testing.assert_allclose(tot / steps, 10.0 * np.array([8, 16, 4, 16]) / 44, rtol=0.06)
    _, per = pyoracle.inner_injection(g, 2, 10.0, 0, 2.0, 1.0, 0.0, EF, 3, 77)
    assert per[3] == 0
