"""Whole steps of the cycle (MainProg order: densities, FFT_X, E, electron push, ion push, MCC, RCX, appends):
the FP64 device cycle against the oracle's cycle, determinism of the fixed-point deposit under re-sorting, and
the fused collision epilogue against the separate collision passes."""
import numpy as np
import pytest

import pyoracle
from edipic_b200 import ELECTRONS, FIELD_ACC_EX, FIELD_PHI, IONS, PREC_FP64, PREC_MIXED, Simulation
from gpu_common import match_by_id, oracle_geom, periodic_dx, random_particles, small_deck


def _plasma(sim, precision, n_per_cell=16, seed=21):
    p = sim.params
    n = p.ncx * p.ncy * n_per_cell
    e = random_particles(sim, n, seed=seed, precision=precision, fast_fraction=0.01)
    ivs = np.random.default_rng(seed + 1).normal(0, 0.0005, (3, n))
    if precision == PREC_MIXED:
        ivs = ivs.astype(np.float32).astype(np.float64)
    sim.upload_particles(ELECTRONS, *e, ids=np.arange(n, dtype=np.uint32))
    sim.upload_particles(IONS, e[0], e[1], ivs[0], ivs[1], ivs[2], ids=np.arange(n, dtype=np.uint32))
    return e, ivs


def _split(d, n):
    """(original particles, particles born during the run) of a downloaded or oracle column set"""
    old = d["id"] < n
    return {k: v[old] for k, v in d.items()}, {k: v[~old] for k, v in d.items()}


def _rows(d):
    r = np.stack([d[k] for k in ("x", "y", "vx", "vy", "vz")], axis=1)
    return r[np.lexsort(r.T[::-1])]


@pytest.mark.gpu
def test_fp64_cycle_matches_oracle_cycle(tmp_path):
    """Two whole FP64 steps against the oracle's cycle. After step 1 the collision counts and every particle agree,
    including the electrons and ions born by ionisation, which join their arrays at the end of the step they are
    born in (pic2d_MainProgram.f90:300, :363). Born particles are numbered in append order (atomic on the device),
    so they are compared as a set of rows. After step 2 the original particles still agree: the step-2 field saw
    the same born particles at the same places, and the original particles' random streams depend only on their
    own ids."""
    d = small_deck(tmp_path, "periodic", ncx=32, ncy=32, n_gas=5.0e22)
    with Simulation(d, precision=PREC_FP64, seed=3) as sim:
        p = sim.params
        e, ivs = _plasma(sim, PREC_FP64, n_per_cell=24)
        n = e[0].size
        oc = pyoracle.OracleCycle(d, e, (e[0], e[1], ivs[0], ivs[1], ivs[2]), seed=3)
        for step in (1, 2):
            sim.step(1)
            oc.step(1)
            c = sim.counters()
            ge, gi = sim.download_particles(ELECTRONS), sim.download_particles(IONS)
            counters, pe, pi = oc.counters, oc.pe, oc.pi
            if step == 1:
                assert min(counters[:3]) > 0 and counters[2] > 0
                assert list(c.en_collisions[:3]) == list(counters[:3])
                assert c.rcx_collisions[0] == counters[4]
                assert c.n_particles[0] == pe.n and c.n_particles[1] == pi.n
            for got, ref in ((ge, pe.arrays()), (gi, pi.arrays())):
                a, a_born = _split(got, n)
                b, b_born = _split(ref, n)
                ia, ib = match_by_id(a, b)
                assert np.abs(periodic_dx(a["x"][ia] - b["x"][ib], p.ncx)).max() < 1e-9
                assert np.abs(a["y"][ia] - b["y"][ib]).max() < 1e-9
                for k in ("vx", "vy", "vz"):
                    assert np.abs(a[k][ia] - b[k][ib]).max() < 1e-9
                if step == 1:
                    assert a_born["x"].size == b_born["x"].size > 0
                    ra, rb = _rows(a_born), _rows(b_born)
                    ra[:, 0] = np.mod(ra[:, 0], p.ncx)
                    rb[:, 0] = np.mod(rb[:, 0], p.ncx)
                    ra, rb = ra[np.lexsort(ra.T[::-1])], rb[np.lexsort(rb.T[::-1])]
                    assert np.abs(ra - rb).max() < 1e-9


@pytest.mark.gpu
def test_sorting_does_not_change_the_state(tmp_path):
    """The fixed-point deposit is order independent and the push is per particle, so the state after several steps
    with periodic re-sorting is bit-identical to the unsorted run."""
    d = small_deck(tmp_path, "periodic", ncx=64, ncy=48, collisions=False, bx=86.6, by=50.0)
    out = []
    for sort_every in (0, 3):
        with Simulation(d, precision=PREC_MIXED, sort_every=sort_every) as sim:
            _plasma(sim, PREC_MIXED, n_per_cell=20)
            sim.step(10)
            out.append((sim.download_particles(ELECTRONS), sim.download_particles(IONS),
                        sim.gather_electron_charge_density(), sim.counters()))
    (e0, i0, r0, c0), (e1, i1, r1, c1) = out
    assert np.array_equal(r0, r1)
    for a, b in ((e0, e1), (i0, i1)):
        ia, ib = match_by_id(a, b)
        for k in ("x", "y", "vx", "vy", "vz"):
            assert np.array_equal(a[k][ia], b[k][ib])
    assert list(c0.electron_hits) == list(c1.electron_hits)


@pytest.mark.gpu
def test_sort_in_the_push_equals_the_separate_sort(tmp_path):
    """A periodic sort done by the next push (each particle written straight to its sorted slot, keyed by its cell
    before the push) and the separate sort pass at the end of the step give bit-identical particles, densities and
    wall hits over 14 steps with a sort every 3, with the unsorted tail of appended particles (ion-induced emission)
    and with particles absorbed in the sorting push."""
    d = small_deck(tmp_path, "periodic", ncx=64, ncy=48, en_collisions=False, rcx=True, bx=86.6, by=50.0,
                   ion_emission=(0.5, 0.0, 10000.0, 2.0))
    out = []
    for fused in (0, 1):
        with Simulation(d, precision=PREC_MIXED, sort_every=3, seed=17) as sim:
            sim._check(sim.lib.edp_set_sort_in_push(sim.ctx, fused), "edp_set_sort_in_push")
            n = 64 * 48 * 20
            e = random_particles(sim, n, seed=61, fast_fraction=0.05)
            ivs = np.random.default_rng(62).normal(0, 0.02, (3, n)).astype(np.float32).astype(np.float64)
            sim.upload_particles(ELECTRONS, *e, ids=np.arange(n, dtype=np.uint32))
            sim.upload_particles(IONS, e[0], e[1], ivs[0], ivs[1], ivs[2], ids=np.arange(n, dtype=np.uint32))
            sim.step(14)
            c = sim.counters()
            out.append((_rows(sim.download_particles(ELECTRONS)), sim.download_particles(IONS),
                        sim.gather_electron_charge_density(), sim.gather_ion_charge_density(),
                        list(c.electron_hits), list(c.ion_hits), c.rcx_collisions[0], list(c.n_particles[:2])))
    (a, b) = out
    assert a[4:] == b[4:] and sum(a[5][:2]) > 100
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
    ia, ib = match_by_id(a[1], b[1])
    for k in ("x", "y", "vx", "vy", "vz"):
        assert np.array_equal(a[1][k][ia], b[1][k][ib]), k


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_fused_collisions_equal_separate_passes(tmp_path, precision):
    d = small_deck(tmp_path, "periodic", ncx=64, ncy=48, n_gas=1.0e23)
    out = []
    later = []
    for fuse in (False, True):
        with Simulation(d, precision=precision, sort_every=4, fuse_collisions=fuse, seed=11) as sim:
            _plasma(sim, precision, n_per_cell=20)
            # one step compares exactly; afterwards particles born by ionisation are numbered in append order,
            # which selects their random streams, so the two runs agree statistically
            sim.step(1)
            c = sim.counters()
            out.append((sim.download_particles(ELECTRONS), list(c.en_collisions[:3]), c.rcx_collisions[0],
                        list(c.n_particles[:2])))
            sim.step(5)
            later.append(np.array(sim.counters().en_collisions[:3], dtype=float))
    (a, ca, ra, na), (b, cb, rb, nb) = out
    assert ca == cb and ra == rb and na == nb
    assert min(ca) > 0
    assert np.all(np.abs(later[0] - later[1]) <= 5.0 * np.sqrt(later[0]) + 5)
    keep_a, keep_b = a["id"] < 64 * 48 * 20, b["id"] < 64 * 48 * 20
    a = {k: v[keep_a] for k, v in a.items()}
    b = {k: v[keep_b] for k, v in b.items()}
    ia, ib = match_by_id(a, b)
    for k in ("vx", "vy", "vz"):
        assert np.abs(a[k][ia] - b[k][ib]).max() < 1e-6


def _oracle_phi(oc, sim):
    """the oracle's potential of its last step on the product's reference node layout"""
    ny, nx = pyoracle.nodes_shape(oc.c.geom)
    nn = nx * ny
    phi = oc.work[3 * nn:4 * nn].reshape(ny, nx)
    out = np.zeros((sim.ny_ref, sim.nx_ref))
    w = min(nx, sim.nx_ref)
    out[:, :w] = phi[:, :w]
    if sim.periodic:
        p = sim.params
        out[:, p.ncx] = out[:, 0]
        out[:, p.ncx + 1] = out[:, 1]
    return out


def _oracle_acc(oc, sim):
    ny, nx = pyoracle.nodes_shape(oc.c.geom)
    nn = nx * ny
    return oc.work[7 * nn:8 * nn].reshape(ny, nx)


@pytest.mark.gpu
def test_mixed_cycle_matches_oracle_cycle_over_12_steps(tmp_path):
    """Twelve whole steps of the mixed-precision cycle (int32 cell + FP32 offsets and velocities, FP32 E, int64
    fixed-point densities, FP64 FFT_X) in the magnetised cfg1 field against the FP64 oracle's cycle, both started
    from the same FP32-snapped particles, collisions off, with a re-sort every 4 steps. The oracle reads the deck
    itself (its constants are not the product's). Stated bounds after 12 steps: positions 2e-5 cell, velocities
    2e-5 of max|v|, potential 1e-5 of max|phi|; identical particle counts and wall hits."""
    d = small_deck(tmp_path, "periodic", ncx=64, ncy=40, collisions=False, rcx=False, bx=86.6, by=50.0,
                   wall_potentials={2: 15.0, 4: -5.0})
    with Simulation(d, precision=PREC_MIXED, sort_every=4, seed=5) as sim:
        p = sim.params
        e, ivs = _plasma(sim, PREC_MIXED, n_per_cell=16, seed=31)
        oc = pyoracle.OracleCycle(d, e, (e[0], e[1], ivs[0], ivs[1], ivs[2]), seed=5)
        sim.step(12)
        oc.step(12)
        c = sim.counters()
        assert c.n_particles[0] == oc.pe.n and c.n_particles[1] == oc.pi.n
        assert list(c.electron_hits[:4]) == list(oc.counters[8:12])
        for got, ref in ((sim.download_particles(ELECTRONS), oc.pe.arrays()),
                         (sim.download_particles(IONS), oc.pi.arrays())):
            ia, ib = match_by_id(got, ref)
            dx = np.abs(periodic_dx(got["x"][ia] - ref["x"][ib], p.ncx)).max()
            dy = np.abs(got["y"][ia] - ref["y"][ib]).max()
            assert dx < 2e-5 and dy < 2e-5, (dx, dy)
            vmax = max(np.abs(ref[k]).max() for k in ("vx", "vy", "vz"))
            dv = max(np.abs(got[k][ia] - ref[k][ib]).max() for k in ("vx", "vy", "vz"))
            assert dv < 2e-5 * vmax, (dv, vmax)
        phi = sim.field(FIELD_PHI)
        ref_phi = _oracle_phi(oc, sim)
        assert np.abs(phi - ref_phi).max() < 1e-5 * np.abs(ref_phi).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_subcycled_ions_match_oracle_cycle(tmp_path, precision):
    """N_subcycles = 3 (ADVANCE_IONS on acc_E with QM2sNsub and X += V N_subcycles, pic2d_IonDynamics.f90:86-155;
    MCC and RCX only on ion steps, pic2d_MainProgram.f90:196-303; CLEAR_ACCUMULATED_FIELDS after them), with the
    ions feeling B and Ez. Against the oracle's subcycled cycle: acc_E after the first two electron steps, acc_E
    cleared after the ion step, and every particle after 3 and 6 steps. FP64 to 1e-9; mixed (FP32 storage, no
    collisions) to 2e-5."""
    fp64 = precision == PREC_FP64
    d = small_deck(tmp_path, "periodic", ncx=32, ncy=32, n_subcycles=3, collisions=fp64, rcx=fp64, n_gas=5.0e22,
                   bx=86.6, by=50.0, ez=200.0, ions_sense_b=True, ions_sense_ez=True)
    tol = 1e-9 if fp64 else 2e-5
    with Simulation(d, precision=precision, sort_every=0, seed=9) as sim:
        p = sim.params
        assert p.n_subcycles == 3 and p.ions_sense_b == 1 and p.ions_sense_ez == 1
        n = p.ncx * p.ncy * 20
        e = random_particles(sim, n, seed=41, precision=precision, fast_fraction=0.01)
        ivs = np.random.default_rng(42).normal(0, 0.01, (3, n))   # ions fast enough that 3 steps move them visibly
        if not fp64:
            ivs = ivs.astype(np.float32).astype(np.float64)
        sim.upload_particles(ELECTRONS, *e, ids=np.arange(n, dtype=np.uint32))
        sim.upload_particles(IONS, e[0], e[1], ivs[0], ivs[1], ivs[2], ids=np.arange(n, dtype=np.uint32))
        oc = pyoracle.OracleCycle(d, e, (e[0], e[1], ivs[0], ivs[1], ivs[2]), seed=9)
        ions0 = sim.download_particles(IONS)
        sim.step(2)
        oc.step(2)
        # two electron steps: acc_E holds E of both, the ions have not moved
        acc = sim.field(FIELD_ACC_EX)
        ref_acc = _oracle_acc(oc, sim)
        w = ref_acc.shape[1]
        assert np.abs(acc[:, :w] - ref_acc).max() <= (1e-12 if fp64 else 1e-6) * np.abs(ref_acc).max()
        ions2 = sim.download_particles(IONS)
        ia, ib = match_by_id(ions2, ions0)
        assert np.array_equal(ions2["x"][ia], ions0["x"][ib])
        for step in (3, 6):
            sim.step(1 if step == 3 else 3)
            oc.step(1 if step == 3 else 3)
            if step == 3:
                assert np.abs(sim.field(FIELD_ACC_EX)).max() == 0.0   # CLEAR_ACCUMULATED_FIELDS
                c = sim.counters()
                if fp64:
                    assert list(c.en_collisions[:3]) == list(oc.counters[:3]) and min(c.en_collisions[:3]) > 0
                    assert c.rcx_collisions[0] == oc.counters[4] > 0
            for got, ref in ((sim.download_particles(ELECTRONS), oc.pe.arrays()),
                             (sim.download_particles(IONS), oc.pi.arrays())):
                a, _ = _split(got, n)
                b, _ = _split(ref, n)
                ia, ib = match_by_id(a, b)
                assert np.abs(periodic_dx(a["x"][ia] - b["x"][ib], p.ncx)).max() < tol, step
                assert np.abs(a["y"][ia] - b["y"][ib]).max() < tol, step
                vmax = max(np.abs(b[k]).max() for k in ("vx", "vy", "vz"))
                for k in ("vx", "vy", "vz"):
                    assert np.abs(a[k][ia] - b[k][ib]).max() < tol * max(1.0, vmax), (step, k)


@pytest.mark.gpu
@pytest.mark.parametrize("ion_emission", [False, True])
def test_push_kernels_give_identical_states(tmp_path, ion_emission):
    """The five kernels of the mixed push over the sorted chunks (one CTA per chunk with the threads' own loads, 4 or 2
    particles per thread, or 4 with each thread's next group copied ahead by cp.async; the persistent streaming kernels whose particle columns arrive by bulk copies, 4 particles
    per thread in 2 stages or 2 in 3 stages) give bit-identical particles, densities, wall hits and charge-exchange counts over 12 steps of the
    magnetised cycle with RCX (the id column in the stages) and, in the second case, ion-induced emission whose
    electrons join after the last sort (the unsorted tail). Particles born on the device take ids in the order of
    atomic appends, which no kernel fixes, so electrons are compared as sets of rows; their physics does not depend
    on the ids without electron-neutral collisions."""
    kw = dict(ion_emission=(0.5, 0.0, 10000.0, 2.0)) if ion_emission else {}
    d = small_deck(tmp_path, "periodic", ncx=128, ncy=64, en_collisions=False, rcx=True, bx=86.6, by=50.0, **kw)
    out = []
    for kind in (0, 1, 2, 3, 4):
        with Simulation(d, precision=PREC_MIXED, sort_every=5, seed=13) as sim:
            sim._check(sim.lib.edp_set_push_kernel(sim.ctx, kind), "edp_set_push_kernel")
            n = 128 * 64 * 24
            e = random_particles(sim, n, seed=51, fast_fraction=0.01)
            ivs = np.random.default_rng(52).normal(0, 0.02, (3, n)).astype(np.float32).astype(np.float64)
            sim.upload_particles(ELECTRONS, *e, ids=np.arange(n, dtype=np.uint32))
            sim.upload_particles(IONS, e[0], e[1], ivs[0], ivs[1], ivs[2], ids=np.arange(n, dtype=np.uint32))
            sim.step(12)
            c = sim.counters()
            out.append((_rows(sim.download_particles(ELECTRONS)), sim.download_particles(IONS),
                        sim.gather_electron_charge_density(), sim.gather_ion_charge_density(),
                        list(c.electron_hits), list(c.ion_hits), c.rcx_collisions[0], list(c.n_particles[:2])))
    ref = out[0]
    assert ref[6] > 0
    assert sum(ref[5][:2]) > 100   # ions reached the walls (and emitted, in the second case)
    for got in out[1:]:
        assert got[4:] == ref[4:]
        assert np.array_equal(got[2], ref[2]) and np.array_equal(got[3], ref[3])
        assert np.array_equal(got[0], ref[0])
        ia, ib = match_by_id(got[1], ref[1])
        for k in ("x", "y", "vx", "vy", "vz"):
            assert np.array_equal(got[1][k][ia], ref[1][k][ib]), k
