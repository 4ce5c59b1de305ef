"""Long-run statistics of the mixed-precision cycle against the plain FP64 device cycle on the RF-driven periodic
configuration (cfg4 physics, reduced to 64 x 64 cells, 64 particles per cell and 400 steps), over 8 seeds: the EEDF
(device energy histogram), the electron and ion density profiles, the electron f(v_x) and the ion flux to each wall
agree within the statistical error across the seeds (Welch z-scores). Both precisions start from the same seed, so
the per-seed differences are also tested (paired): their mean is so well resolved (relative biases of 1e-4 show)
that the paired test is an equivalence test, asking that no component's bias exceed 1 % of its value by more than
6 standard errors (t-distribution with 7 degrees of freedom), and it states the smallest relative bias it could
detect."""
import numpy as np
import pytest

from edipic_b200 import ELECTRONS, PREC_FP64, PREC_MIXED, Simulation, decks
from edipic_b200.longrun import compare, compare_paired, run


@pytest.mark.gpu
def test_mixed_matches_fp64_statistically(tmp_path):
    kw = dict(steps=400, cells=(64, 64), ppc=64, burn_in=200, sample_every=20, workdir=str(tmp_path))
    mixed = [run(PREC_MIXED, 1000 + s, **kw) for s in range(8)]
    fp64 = [run(PREC_FP64, 1000 + s, **kw) for s in range(8)]
    welch = compare(mixed, fp64)
    paired = compare_paired(mixed, fp64, rel_tol=0.01)
    for k, v in paired.items():
        if k == "ion_flux" and v["n"] == 0:
            # few ions reach the walls in 200 steps: the two precisions may count exactly the same in every seed
            assert all(a["ion_flux"] == b["ion_flux"] for a, b in zip(mixed, fp64))
            continue
        assert v["n"] > 0, k
        assert v["max_excess_z"] < 6.0, (k, v)
        w = welch[k]
        assert w["max_abs_z"] < 5.0 and w["mean_z2"] < 2.0, (k, w)
    # the pairing makes the comparison sensitive: biases of a few percent of the EEDF or the density would show
    assert paired["eedf"]["detectable_bias_median"] < 0.05 and paired["ne"]["detectable_bias_median"] < 0.05, paired
    assert min(r["ion_flux"][0] + r["ion_flux"][1] for r in mixed) > 0


@pytest.mark.gpu
def test_energy_histogram_matches_downloaded_particles(tmp_path):
    """edp_energy_histogram against numpy on the downloaded electrons and ions (mixed and FP64)."""
    d = decks.write_deck(str(tmp_path), "cfg4", ncx=64, ncy=32, ppc=16)
    edges = np.concatenate([[0.0], np.geomspace(0.05, 100.0, 40)])
    for prec in (PREC_MIXED, PREC_FP64):
        with Simulation(d, precision=prec, seed=3) as sim:
            sim.distribute_particles(16)
            sim.step(3)
            ef = sim.deck.tables.energy_factor_eV
            for sp, f in ((ELECTRONS, ef), (1, ef * sim.params.ion_mass_me[0])):
                got = sim.energy_histogram(sp, edges)
                p = sim.download_particles(sp)
                e = (p["vx"] ** 2 + p["vy"] ** 2 + p["vz"] ** 2) * f
                want, _ = np.histogram(e[(e >= edges[0]) & (e < edges[-1])], bins=edges)
                # a particle exactly on an edge may fall on either side by the last bit of the energy
                assert np.abs(got - want).sum() <= 2 and got.sum() > 0.5 * len(e), (prec, sp)
