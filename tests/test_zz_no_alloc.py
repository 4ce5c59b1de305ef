"""The allocation-free FFT_X solve, edp_poisson_fftx_noalloc, for callers that cannot allocate device memory
(their GPU memory belongs to another runtime or pool): it takes the caller's device buffers and keeps its
workspace in a fixed file-scope device array. Checked through the C ABI against the context-based solve
(edp_field_fftx) on the same charge density, on two calls in a row, to the FP64 tolerance of the FFT_X tests."""
import ctypes as C

import numpy as np
import pytest

from gpu_common import random_particles, small_deck


@pytest.mark.gpu
def test_noalloc_fftx_matches_context_solve(tmp_path):
    import torch

    from edipic_b200 import ELECTRONS, FIELD_RHO_TOTAL, IONS, Simulation, library
    lib = library()
    d = small_deck(tmp_path, "periodic", ncx=128, ncy=96, wall_potentials={2: 25.0, 4: -5.0})
    with Simulation(d, sort_every=0) as sim:
        p = sim.params
        n_e, n_i = 128 * 96 * 8, 128 * 96 * 4
        for call in range(2):
            sim.upload_particles(ELECTRONS, *random_particles(sim, n_e, seed=10 + call))
            sim.upload_particles(IONS, *random_particles(sim, n_i, seed=20 + call, vscale=0.001))
            phi_ref = sim.solve_poisson_fftx_linsysy(want_phi=True)
            rho = sim.field(FIELD_RHO_TOTAL)
            assert np.abs(rho).max() > 0
            rho_d = torch.from_numpy(np.ascontiguousarray(rho)).cuda()
            phi_d = torch.full_like(rho_d, float("nan"))
            torch.cuda.synchronize()
            rc = lib.edp_poisson_fftx_noalloc(p.ncx, p.ncy, C.c_void_p(rho_d.data_ptr()), p.wall_phi_const[0],
                                              p.wall_phi_const[1], C.c_void_p(phi_d.data_ptr()), None)
            assert rc == 0
            torch.cuda.synchronize()
            phi = phi_d.cpu().numpy()
            assert np.isfinite(phi).all()
            assert np.abs(phi - phi_ref).max() <= 1e-12 * np.abs(phi_ref).max(), call
        # a grid whose workspace exceeds the fixed array is refused before any work is queued
        big = torch.zeros(8, dtype=torch.float64, device="cuda")
        rc = lib.edp_poisson_fftx_noalloc(4096, 4095, C.c_void_p(big.data_ptr()), 0.0, 0.0,
                                          C.c_void_p(big.data_ptr()), None)
        assert rc == -3
