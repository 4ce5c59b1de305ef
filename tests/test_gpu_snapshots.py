"""CREATE_SNAPSHOT from device moments and histograms (edipic_b200.snapshots): on a freshly distributed Maxwellian
plasma the density file gives the deck's initial density and the temperature files its initial temperatures at
interior nodes (the ions' z temperature is zero: they start with vz = 0); the potential and VDF files hold exactly the device arrays they were made from, the density file the
device moments to FP32 rounding."""
import numpy as np
import pytest

from edipic_b200 import ELECTRONS, FIELD_PHI, PREC_MIXED, Simulation, snapshots
from gpu_common import small_deck


@pytest.mark.gpu
@pytest.mark.parametrize("geometry", ["periodic", "walled"])
def test_snapshot_files(tmp_path, geometry):
    d = small_deck(tmp_path / "deck", geometry, ncx=64, ncy=64, ppc=400, **({"inner": False} if geometry == "walled" else {}))
    out = tmp_path / "snap"
    out.mkdir()
    with Simulation(d, precision=PREC_MIXED, sort_every=4, fuse_collisions=False) as sim:
        sim.distribute_particles(400)
        vdf = dict(nbox=(2, 2), n_max_vel_e=4, n_vbins_e=10, n_max_vel_i=4, n_vbins_i=10, two_d=True)
        files = snapshots.create_snapshot(sim, 7, str(out), vdf=vdf)
        m = sim.collect_moments(ELECTRONS)
        phi = sim.field(FIELD_PHI)
        e1, e2, _ = sim.calculate_vdf(ELECTRONS, (2, 2), 4, 10, True)
        deck = sim.deck
        p = sim.params
    names = {f.split("/")[-1] for f in files}
    assert len(names) == 38 + 2 and "_0007_Ni_1_m3_2D.bin" in names and "_0007_vdf2d.bin" in names
    sc = snapshots.scales(sim)
    _, _, ne = snapshots.read_2d(out / "_0007_Ne_m3_2D.bin")
    # moments are FP32 atomic sums: two calls agree to rounding, not bit for bit
    ref = m[0] * np.float32(sc["N_scale_part_m3"])
    assert np.abs(ne - ref).max() <= 1e-5 * np.abs(ref).max()
    _, _, f = snapshots.read_2d(out / "_0007_F_V_2D.bin")
    assert np.array_equal(f, (phi * p.f_scale_v).astype(np.float32))
    inner = (slice(4, -4), slice(4, -4))
    assert abs(np.mean(ne[inner]) / deck.init_ne_m3 - 1.0) < 0.02
    for c in "XYZ":
        _, _, t = snapshots.read_2d(out / f"_0007_T{c}e_eV_2D.bin")
        assert abs(np.mean(t[inner]) / deck.init_te_ev - 1.0) < 0.03, (c, np.mean(t[inner]), deck.init_te_ev)
        _, _, ti = snapshots.read_2d(out / f"_0007_T{c}i_1_eV_2D.bin")
        if c == "Z":   # DISTRIBUTE_PARTICLES starts the ions with vz = 0 (pic2d_CurProblemValues.f90:3298)
            assert np.all(ti == 0.0)
        else:
            assert abs(np.mean(ti[inner]) / deck.init_ti_ev[0] - 1.0) < 0.05, (c, np.mean(ti[inner]))
    raw = np.fromfile(out / "_0007_vdf2d.bin", dtype=np.int32)
    rl = 80
    one = 4 + rl * rl
    for n in range(4):
        s0 = 6 + n * one
        assert np.array_equal(raw[s0 + 4:s0 + one], e2[n].ravel())
    raw1 = np.fromfile(out / "_0007_vdf1d.bin", dtype=np.int32)
    s0 = 9 + 1 + p.n_ion_species
    assert np.array_equal(raw1[s0 + 4:s0 + 4 + rl], e1[0, 0])
