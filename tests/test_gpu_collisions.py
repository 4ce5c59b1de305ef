"""Electron-neutral MCC and Ar+-Ar charge exchange on the device against the oracle fed with the same Philox
variates: kind selection bit for bit (PERFORM_ELECTRON_NEUTRAL_COLLISIONS :451-485), per-kind counts, post-
collision velocities, ionisation products, RCX decisions and Maxwellian replacements."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import ELECTRONS, IONS, PREC_FP64, PREC_MIXED, Simulation
from gpu_common import match_by_id, small_deck


def _mcc_setup(sim, d):
    p, t = sim.params, sim.deck.tables
    neu = pyoracle.read_neutral_deck(d)
    ot = pyoracle.MccTables(neu, p.n_subcycles, p.delta_t_s)
    return neu, ot


@pytest.mark.gpu
def test_kind_choice_bit_exact(tmp_path):
    d = small_deck(tmp_path, "periodic")
    with Simulation(d) as sim:
        neu, ot = _mcc_setup(sim, d)
        rng = np.random.default_rng(5)
        n = 200000
        e = np.exp(rng.uniform(np.log(1e-4), np.log(5e3), n))
        r = rng.random(n)
        # edge cases: every table energy, segment boundaries, energies just around them, r on table values
        tab_e = ot.energy.copy()
        e = np.concatenate([e, tab_e, np.nextafter(tab_e, 0), np.nextafter(tab_e, 1e9), [0.0, 1e-30, 1e6]])
        P = ot.prob.reshape(-1, 3)
        r_tab = P[rng.integers(0, P.shape[0], e.size - n), rng.integers(0, 3, e.size - n)]
        r = np.concatenate([r, r_tab])
        got = sim.mcc_choose(e, r)
    ref = ot.choose(e, r)
    assert np.array_equal(got, ref)
    assert set(np.unique(ref)) == {1, 2, 3, 4}


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_mcc_pass_matches_oracle(tmp_path, precision):
    d = small_deck(tmp_path, "periodic", n_gas=2.0e23)
    with Simulation(d, precision=precision, fuse_collisions=False, sort_every=0, seed=77) as sim:
        p = sim.params
        neu, ot = _mcc_setup(sim, d)
        rng = np.random.default_rng(9)
        n = 200000
        x = rng.uniform(0, p.ncx, n)
        y = rng.uniform(0.5, p.ncy - 0.5, n)
        # speeds spanning 0.01 .. 200 eV
        en = np.exp(rng.uniform(np.log(0.01), np.log(200.0), n))
        speed = np.sqrt(en / sim.deck.tables.energy_factor_eV)
        u = rng.normal(size=(3, n))
        u /= np.linalg.norm(u, axis=0)
        v = speed * u
        if precision == PREC_MIXED:
            i, j = np.floor(x), np.floor(y)
            x = i + (x - i).astype(np.float32)
            y = j + (y - j).astype(np.float32)
            v = v.astype(np.float32).astype(np.float64)
        ids = np.arange(n, dtype=np.uint32)
        sim.upload_particles(ELECTRONS, x, y, v[0], v[1], v[2], ids=ids)
        sim.upload_particles(IONS, x[:1000], y[:1000], v[0, :1000] * 0, v[1, :1000] * 0, v[2, :1000] * 0,
                             ids=np.arange(1000, dtype=np.uint32))
        cnt = sim.perform_electron_neutral_collisions()
        got = sim.download_particles(ELECTRONS)
        sim.end_ion_cycle()
        ions = sim.download_particles(IONS)
    ps = pyoracle.ParticleSet(x, y, v[0], v[1], v[2], ids=ids)
    be = pyoracle.ParticleSet(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), cap=n)
    bi = pyoracle.ParticleSet(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), cap=n)
    import ctypes as C
    mv, _ = pyoracle.maxwell_tables()
    t = sim.deck.tables
    ctx = pyoracle.MccCtx(77, 0, t.energy_factor_eV, t.neutral_mass_amu, t.ion_velocity_factor[2], pyoracle.dp(mv))
    counters = np.zeros(8, dtype=np.int64)
    pyoracle.lib().oracle_mcc_philox(C.byref(ot.t), C.byref(ctx), C.byref(ps.s), C.byref(be.s), C.byref(bi.s), n,
                                     counters.ctypes.data_as(pyoracle._I64))
    assert np.array_equal(cnt[:3], counters[:3]), (cnt, counters)
    assert counters[:3].min() > 100
    ref = ps.arrays()
    ia, ib = match_by_id(got, ref)
    tol = 2e-6 if precision == PREC_MIXED else 1e-12
    vmax = np.abs(v).max()
    for k in ("vx", "vy", "vz"):
        assert np.abs(got[k][ia] - ref[k][ib]).max() <= tol * vmax
    # ions born by ionisation (appended after the collisions, PROCESS_ADDED_IONS)
    new = ions["id"] >= 1000
    assert new.sum() == bi.n == counters[2]
    gi = np.stack([ions[k][new] for k in ("x", "y", "vx", "vy", "vz")])
    ri = bi.arrays()
    rk = np.stack([ri[k] for k in ("x", "y", "vx", "vy", "vz")])
    order_g = np.lexsort(gi[::-1])
    order_r = np.lexsort(rk[::-1])
    assert np.allclose(gi[:, order_g], rk[:, order_r], rtol=0, atol=1e-6 if precision == PREC_MIXED else 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_rcx_pass_matches_oracle(tmp_path, precision):
    d = small_deck(tmp_path, "periodic", n_gas=2.0e23)
    with Simulation(d, precision=precision, fuse_collisions=False, sort_every=0, seed=5) as sim:
        p, t = sim.params, sim.deck.tables
        rng = np.random.default_rng(3)
        n = 200000
        x = rng.uniform(0, p.ncx, n)
        y = rng.uniform(0.5, p.ncy - 0.5, n)
        v = rng.normal(0, 0.003, (3, n))
        if precision == PREC_MIXED:
            i, j = np.floor(x), np.floor(y)
            x = i + (x - i).astype(np.float32)
            y = j + (y - j).astype(np.float32)
            v = v.astype(np.float32).astype(np.float64)
        ids = np.arange(n, dtype=np.uint32) + 100
        sim.upload_particles(ELECTRONS, x[:10], y[:10], v[0, :10], v[1, :10], v[2, :10])
        sim.upload_particles(IONS, x, y, v[0], v[1], v[2], ids=ids)
        count = sim.perform_resonant_charge_exchange()
        got = sim.download_particles(IONS)
    mv, _ = pyoracle.maxwell_tables()
    r = pyoracle.Rcx(t.rcx_prob_factor, p.v_scale_ms, p.ion_mass_me[0] * t.energy_factor_eV, t.rcx_sigma_1eV,
                     t.rcx_alpha, t.rcx_probab_thermal[0], t.rcx_vfactor[0])
    ctx = pyoracle.MccCtx(5, 0, t.energy_factor_eV, t.neutral_mass_amu, 0.0, pyoracle.dp(mv))
    ps = pyoracle.ParticleSet(x, y, v[0], v[1], v[2], ids=ids)
    import ctypes as C
    ref_count = pyoracle.lib().oracle_rcx_philox(C.byref(r), C.byref(ctx), 0, C.byref(ps.s))
    assert count == ref_count and ref_count > 100
    ref = ps.arrays()
    ia, ib = match_by_id(got, ref)
    for k in ("vx", "vy", "vz"):
        assert np.abs(got[k][ia] - ref[k][ib]).max() <= (1e-9 if precision == PREC_MIXED else 1e-15)
