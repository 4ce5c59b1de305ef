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
