"""The oracle's electron-induced emission (oracle_see, restating pic2d_SEEmission.f90:4-1208) against properties the
reference's algorithm fixes: the classic coefficient equals its maximum at E_max and normal incidence, so the mean
number of true secondaries there is maxD (1 - fractions); specular reflection mirrors the normal component; random
elastic reflection and inelastic backscattering leave with cos(theta) = sqrt(1 - R^2) (mean pi/4) and, for the
inelastic case, an energy uniform in (0, E) (mean E/2); nothing below the lowest threshold; elastic + inelastic
above 1 is reported."""
import numpy as np

import pyoracle
from edipic_b200.decks import SEE_OFF

EF = 1000.0
XMAX, YMAX = 64.0, 48.0


def emitter(**kw):
    return pyoracle.ElectronEmission(dict(SEE_OFF, **kw), EF)


def speed(e_ev):
    return np.sqrt(e_ev / EF)


def test_classic_true_yield_at_maximum():
    em = emitter(true_model=2, true_t_ev=2.0, classic_e0_ev=13.0, classic_emax_ev=500.0, classic_max=2.4,
                 classic_k_smooth=1.0, elastic_frac_classic=0.1, inelastic_frac_classic=0.2)
    v = speed(500.0)
    n = [em.emit(0, 10.0, -0.01, 0.0, -v, 0.0, k, 3, 7, XMAX, YMAX)[1] for k in range(20000)]
    expect = 2.4 * (1 - 0.1 - 0.2)   # 1.68: one electron, then a second with probability 0.68
    assert set(n) == {1, 2}
    assert abs(np.mean(n) - expect) < 4 * np.sqrt(0.68 * 0.32 / len(n))
    assert em.emit(0, 10.0, -0.01, 0.0, -speed(12.0), 0.0, 1, 3, 7, XMAX, YMAX)[1] == 0   # below E_see_0


def test_specular_and_random_reflection():
    em = emitter(elastic_model=1, elastic_type=0, elastic_yield=1.0, elastic_emin_ev=0.0, elastic_emax_ev=1e4)
    rows, n = em.emit(3, XMAX + 0.1, 20.0, 0.3, -0.1, 0.05, 9, 3, 7, XMAX, YMAX)
    assert n == 1 and np.allclose(rows[0], [XMAX - 1e-6, 20.0, -0.3, -0.1, 0.05], rtol=0, atol=1e-15)
    em = emitter(elastic_model=1, elastic_type=1, elastic_yield=1.0, elastic_emin_ev=0.0, elastic_emax_ev=1e4)
    v = speed(50.0)
    rows = np.concatenate([em.emit(1, 5.0, YMAX + 0.01, 0.0, v, 0.0, k, 3, 7, XMAX, YMAX)[0] for k in range(20000)])
    sp = np.sqrt((rows[:, 2:] ** 2).sum(1))
    assert np.allclose(sp, v, rtol=1e-12)
    cos = -rows[:, 3] / sp                     # leaving the top wall downwards
    assert np.all(cos >= 0) and abs(cos.mean() - np.pi / 4) < 0.01
    assert np.all(rows[:, 1] == YMAX - 1e-6)


def test_inelastic_backscatter_and_limits():
    em = emitter(inelastic_model=1, inelastic_yield=1.0, inelastic_emin_ev=0.0, inelastic_emax_ev=1e4)
    v = speed(80.0)
    rows = np.concatenate([em.emit(2, -0.1, 7.0, -v, 0.0, 0.0, k, 3, 7, XMAX, YMAX)[0] for k in range(20000)])
    e = (rows[:, 2:] ** 2).sum(1) / v ** 2
    assert abs(e.mean() - 0.5) < 0.01 and np.all(e <= 1.0)
    assert np.all(rows[:, 2] >= 0) and np.all(rows[:, 0] == 1e-6)
    bad = emitter(elastic_model=1, elastic_yield=0.7, elastic_emin_ev=0.0, elastic_emax_ev=1e4,
                  inelastic_model=1, inelastic_yield=0.5, inelastic_emin_ev=0.0, inelastic_emax_ev=1e4)
    assert bad.emit(0, 1.0, -0.01, 0.0, -v, 0.0, 1, 3, 7, XMAX, YMAX)[1] == -1
    low = emitter(true_model=1, true_yield=0.5, true_emin_ev=20.0, true_emax_ev=100.0, true_t_ev=1.0)
    assert low.emit(0, 1.0, -0.01, 0.0, -speed(19.0), 0.0, 1, 3, 7, XMAX, YMAX)[1] == 0
