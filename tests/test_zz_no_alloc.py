"""The allocation-free FFT_X solve, edp_poisson_fftx_noalloc, for callers that cannot allocate device memory
(their GPU memory belongs to another runtime or pool): it takes the caller's device buffers and keeps its
workspace in a fixed file-scope device array. Checked through the C ABI against the context-based solve
(edp_field_fftx) on the same charge density, on two calls in a row, to the FP64 tolerance of the FFT_X tests;
also at the largest 1024-column grid the array holds, at 4096 columns (FFT rows beyond 48 KiB of shared memory),
and the refusal of the first grid that does not fit."""
import ctypes as C

import numpy as np
import pytest

from gpu_common import random_particles, small_deck


def workspace_bytes(ncx, ncy):
    """The workspace the entry point needs: spectrum, elimination coefficients, twiddles, 256-byte sections."""
    a = lambda b: (b + 255) & ~255
    nm = ncx // 2 + 1
    return a(a((ncy + 1) * nm * 16) + (ncy + 1) * nm * 8) + (ncx // 2) * 16


SCRATCH = 16 << 20   # EDP_NOALLOC_SCRATCH_BYTES


def _solve_against_context(tmp_path, ncx, ncy, calls, ppc_e=8, ppc_i=4):
    import torch

    from edipic_b200 import ELECTRONS, FIELD_RHO_TOTAL, IONS, Simulation, library
    lib = library()
    d = small_deck(tmp_path, "periodic", ncx=ncx, ncy=ncy, wall_potentials={2: 25.0, 4: -5.0})
    with Simulation(d, sort_every=0) as sim:
        p = sim.params
        n_e, n_i = ncx * ncy * ppc_e, ncx * ncy * ppc_i
        for call in range(calls):
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
            assert np.abs(phi - phi_ref).max() <= 1e-12 * np.abs(phi_ref).max(), (ncx, ncy, call)


def test_workspace_limits_stated_in_the_header():
    """The largest grids the header names fit the array, and one more row does not."""
    for ncx, ncy in ((512, 2718), (1024, 1360), (2048, 680), (4096, 339)):
        assert workspace_bytes(ncx, ncy) <= SCRATCH < workspace_bytes(ncx, ncy + 1)
    assert workspace_bytes(1024, 1024) <= SCRATCH


@pytest.mark.gpu
def test_noalloc_fftx_matches_context_solve(tmp_path):
    _solve_against_context(tmp_path, 128, 96, calls=2)


@pytest.mark.gpu
def test_noalloc_fftx_at_capacity(tmp_path):
    import torch

    from edipic_b200 import library
    lib = library()
    # the largest 1024-column grid, and 4096 columns (its FFT rows opt in to more than 48 KiB of shared memory)
    _solve_against_context(tmp_path / "a", 1024, 1360, calls=1, ppc_e=2, ppc_i=1)
    _solve_against_context(tmp_path / "b", 4096, 96, calls=2, ppc_e=2, ppc_i=1)
    # the first grids whose workspace exceeds the array are refused before any work is queued
    big = torch.zeros(8, dtype=torch.float64, device="cuda")
    for ncx, ncy in ((1024, 1361), (4096, 340), (4096, 4095)):
        rc = lib.edp_poisson_fftx_noalloc(ncx, ncy, C.c_void_p(big.data_ptr()), 0.0, 0.0,
                                          C.c_void_p(big.data_ptr()), None)
        assert rc == -3, (ncx, ncy)
