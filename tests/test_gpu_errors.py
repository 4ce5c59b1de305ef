"""Error reporting without any device fault: host-side checks and device error words raised by small
capacities or impossible tolerances (fault injection stays on the host)."""
import numpy as np
import pytest

from edipic_b200 import ELECTRONS, EdpError, IONS, PREC_MIXED, Simulation
from gpu_common import random_particles, small_deck


@pytest.mark.gpu
def test_upload_outside_domain_is_rejected(tmp_path):
    d = small_deck(tmp_path, "periodic", ncx=32, ncy=32)
    with Simulation(d) as sim:
        x = np.array([1.0, 5.0, 3.0])
        y = np.array([1.0, 40.0, 3.0])    # y beyond the top wall
        with pytest.raises(EdpError) as e:
            sim.upload_particles(ELECTRONS, x, y, x * 0, x * 0, x * 0)
        assert e.value.code == -4


@pytest.mark.gpu
def test_capacity_too_small_is_rejected(tmp_path):
    d = small_deck(tmp_path, "periodic", ncx=32, ncy=32)
    with Simulation(d, capacity=[100, 100]) as sim:
        x, y, vx, vy, vz = random_particles(sim, 1000)
        with pytest.raises(EdpError) as e:
            sim.upload_particles(ELECTRONS, x, y, vx, vy, vz)
        assert e.value.code == -3


@pytest.mark.gpu
def test_cg_not_converged_reports(tmp_path):
    d = small_deck(tmp_path, "walled", ncx=64, ncy=64)
    with Simulation(d) as sim:
        x, y, vx, vy, vz = random_particles(sim, 50000)
        sim.upload_particles(ELECTRONS, x, y, vx, vy, vz)
        with pytest.raises(EdpError) as e:
            sim.solve_potential_with_cg(rtol=1e-12, max_it=1)
        assert e.value.code == -5
        # the context stays usable
        assert sim.solve_potential_with_cg(rtol=1e-8, max_it=20000) > 1


@pytest.mark.gpu
def test_order_errors(tmp_path):
    d = small_deck(tmp_path, "periodic", ncx=32, ncy=32)
    with Simulation(d) as sim:
        with pytest.raises(EdpError) as e:
            sim.advance_electrons()
        assert e.value.code == -7
        with pytest.raises(EdpError):
            sim.solve_potential_with_cg()


@pytest.mark.gpu
def test_id_range_exhaustion_is_refused(tmp_path):
    """A context whose id range ends 10 ids after its particles: more than 10 ionisations in a step must not take
    ids past the end (they belong to the next rank and would repeat its random streams). The born particles past
    the range are not appended, edp_query_counters reports EDP_ERR_CAPACITY, and no id appears twice."""
    d = small_deck(tmp_path, "periodic", ncx=32, ncy=32, n_gas=5.0e22)
    with Simulation(d, seed=7) as sim:
        n = 32 * 32 * 8
        base = 1000
        sim.set_id_base(base, base + n + 10)
        rng = np.random.default_rng(3)
        x, y = rng.uniform(0, 32, n), rng.uniform(1, 31, n)
        i, j = np.floor(x), np.floor(y)
        x = i + (x - i).astype(np.float32).astype(np.float64)
        y = j + (y - j).astype(np.float32).astype(np.float64)
        v = rng.normal(0.0, 1.0, (3, n))
        v *= (0.2 / np.sqrt((v * v).sum(axis=0)))   # |v| = 0.2 cells/step, about 45 eV: well above the threshold
        v = v.astype(np.float32).astype(np.float64)
        ids = np.arange(base, base + n, dtype=np.uint32)
        sim.upload_particles(ELECTRONS, x, y, v[0], v[1], v[2], ids=ids)
        sim.upload_particles(IONS, x, y, 0 * x, 0 * x, 0 * x, ids=ids)
        with pytest.raises(EdpError) as e:
            sim.step(1)
            sim.counters()
        assert e.value.code == -3
        for sp in (ELECTRONS, IONS):
            got = sim.download_particles(sp, cap=2 * n + 1024)["id"].astype(np.int64)   # the counters stay in error
            assert np.unique(got).size == got.size
            assert got.min() >= base and got.max() < base + n + 10
