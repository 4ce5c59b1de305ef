"""A domain cut into x strips against one context holding the whole domain. The strips push their own
particles against their columns of the whole grid's field, deposit into their own and ghost nodes, sum the densities
into the whole grid and hand the particles that end a step in ghost columns to the neighbour owning them. Without
ionisation (whose new ids depend on the order of creation) the union of the strips' particles, the potential and the
wall-hit counts equal the one-context run bit for bit in mixed precision: the densities are int64 fixed-point sums and
the particles keep their FP32 offsets. Two strips per process on the one test GPU (LocalStrips), and two ranks that
share it through gloo (StripRank: host-side sums and moves, no kernel waits on another)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gpu_common import random_particles, small_deck

STEPS = 12


def _rows(d):
    o = np.argsort(d["id"])
    return np.stack([d[k][o] for k in ("x", "y", "vx", "vy", "vz")], axis=1), d["id"][o], d["tag"][o]


def _plasma(sim, n=30000):
    e = random_particles(sim, n, seed=1)
    i = random_particles(sim, n, seed=2, vscale=0.002)
    ids = np.arange(n, dtype=np.uint32) * 3 + 5
    tags = (np.arange(n) % 7).astype(np.int32)
    return e, i, ids, tags


def _reference(deck, sort_every, steps, n_hits=2):
    from edipic_b200 import ELECTRONS, FIELD_PHI, IONS, Simulation
    with Simulation(deck, sort_every=sort_every, fuse_collisions=True) as sim:
        e, i, ids, tags = _plasma(sim)
        sim.upload_particles(ELECTRONS, *e, tag=tags, ids=ids)
        sim.upload_particles(IONS, *i, tag=tags, ids=ids)
        sim.step(steps)
        c = sim.counters()
        return ((e, i, ids, tags), [sim.download_particles(s) for s in (ELECTRONS, IONS)], sim.field(FIELD_PHI),
                list(c.electron_hits[:n_hits]), list(c.ion_hits[:n_hits]))


@pytest.mark.gpu
@pytest.mark.parametrize("n_strips,sort_every", [(2, 0), (2, 4), (3, 4)])
def test_strips_equal_one_context(tmp_path, n_strips, sort_every):
    from edipic_b200 import ELECTRONS, FIELD_PHI, IONS
    from edipic_b200.strips import LocalStrips
    deck = small_deck(tmp_path, "periodic", collisions=False, bx=86.6, by=50.0, wall_potentials={2: 5.0, 4: -3.0})
    (e, i, ids, tags), ref, phi_ref, eh, ih = _reference(deck, sort_every, STEPS)
    with LocalStrips(deck, n_strips, ghost=4, sort_every=sort_every) as ls:
        ls.load(ELECTRONS, *e, ids=ids, tags=tags)
        ls.load(IONS, *i, ids=ids, tags=tags)
        ls.step(STEPS)
        got = [ls.download(s) for s in (ELECTRONS, IONS)]
        phi = ls.field.field(FIELD_PHI)
        c = ls.counters()
        moved = [s.sim.counters().n_particles[0] for s in ls.strips]
    for s in range(2):
        a, ia, ta = _rows(got[s])
        b, ib, tb = _rows(ref[s])
        assert np.array_equal(ia, ib) and np.array_equal(ta, tb)
        assert np.array_equal(a, b), np.abs(a - b).max()
    assert np.array_equal(phi, phi_ref)
    assert c["electron_hits"][:2] == eh and c["ion_hits"][:2] == ih
    assert sum(eh) > 0 and min(moved) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("n_strips", [2, 3])
def test_walled_strips_equal_one_context(tmp_path, n_strips):
    """The walled domain with the metal rectangle at -100 V across the strip boundary, the field by multigrid PCG on
    the whole grid: the end strips have the domain's walls instead of ghost columns, and the rectangle absorbs in
    every strip it reaches. Same particles and wall hits as one context."""
    from edipic_b200 import ELECTRONS, FIELD_PHI, IONS
    from edipic_b200.strips import LocalStrips
    deck = small_deck(tmp_path, "walled", collisions=False, wall_potentials={2: 5.0, 4: -3.0})
    (e, i, ids, tags), ref, phi_ref, eh, ih = _reference(deck, 4, STEPS, n_hits=8)
    with LocalStrips(deck, n_strips, ghost=4, sort_every=4) as ls:
        assert [s.frames[s.index][:2] for s in ls.strips][0][0] == 0   # the left wall takes no ghost columns
        ls.load(ELECTRONS, *e, ids=ids, tags=tags)
        ls.load(IONS, *i, ids=ids, tags=tags)
        ls.step(STEPS)
        got = [ls.download(s) for s in (ELECTRONS, IONS)]
        phi = ls.field.field(FIELD_PHI)
        c = ls.counters()
    # CG sums its dot products with atomics in an order that varies from run to run, so the potential of two runs
    # agrees to rounding, not to the bit; the FP32 field and the particles almost always do
    for s in range(2):
        a, ia, ta = _rows(got[s])
        b, ib, tb = _rows(ref[s])
        assert np.array_equal(ia, ib) and np.array_equal(ta, tb)
        assert np.abs(a - b).max() < 1e-6
    assert np.abs(phi - phi_ref).max() <= 1e-10 * np.abs(phi_ref).max()
    assert c["electron_hits"] == eh and c["ion_hits"] == ih
    assert eh[2] > 0 and eh[3] > 0 and eh[4] > 0   # left and right walls and the rectangle took electrons


@pytest.mark.gpu
def test_strips_with_collisions_keep_running(tmp_path):
    """With the full collision set the run over strips is the same physics with other ids for the new particles:
    no particle is lost or doubled by the moves (counts against the one-context run within the ionisation noise)."""
    from edipic_b200 import ELECTRONS, IONS, Simulation
    from edipic_b200.strips import LocalStrips
    deck = small_deck(tmp_path, "periodic")
    with Simulation(deck, sort_every=4) as sim:
        e, i, ids, tags = _plasma(sim)
        sim.upload_particles(ELECTRONS, *e, tag=tags, ids=ids)
        sim.upload_particles(IONS, *i, tag=tags, ids=ids)
        sim.step(20)
        ref = sim.counters()
    with LocalStrips(deck, 2, ghost=4, sort_every=4) as ls:
        ls.load(ELECTRONS, *e, ids=ids, tags=tags)
        ls.load(IONS, *i, ids=ids, tags=tags)
        ls.step(20)
        c = ls.counters()
        d = ls.download(ELECTRONS)
    assert len(np.unique(d["id"])) == len(d["id"])
    for s in range(2):
        assert abs(c["n_particles"][s] - ref.n_particles[s]) <= 0.02 * ref.n_particles[s]


@pytest.mark.gpu
def test_strip_api_refusals(tmp_path):
    import ctypes as C
    from edipic_b200 import ELECTRONS, EdpError, Simulation
    deck = small_deck(tmp_path, "periodic", collisions=False)
    with Simulation(deck) as sim:   # the whole periodic domain is not a strip
        with pytest.raises(EdpError):
            sim._check(sim.lib.edp_set_strip(sim.ctx, 4, 4, -4, 64, 1), "edp_set_strip")
        nl, nr = C.c_int64(), C.c_int64()
        assert sim.lib.edp_strip_take(sim.ctx, 0, None, 0, None, 0, C.byref(nl), C.byref(nr)) == -7
    with Simulation(deck, strip=(32, 4, 4, -4)) as st:
        assert st.params.ncx == 40 and not st.periodic
        with pytest.raises(EdpError):   # no wall emission on a strip
            st.set_ion_emission(0, 1, 0.1, 0.0, 100.0, 2.0)
        rec = torch.zeros((1, 8), dtype=torch.float64, device="cuda")
        assert st.lib.edp_strip_put(st.ctx, 0, C.c_void_p(rec.data_ptr()), 1, 0.0) == -7   # before the upload
        x = np.array([10.5])
        st.upload_particles(ELECTRONS, x, x, 0 * x, 0 * x, 0 * x)
        assert st.lib.edp_set_strip(st.ctx, 4, 4, -4, 64, 1) == -7   # after the upload


def _rank_worker(rank, world, port, deck, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from edipic_b200 import ELECTRONS, FIELD_PHI, IONS, Simulation
    from edipic_b200.strips import StripRank
    try:
        with Simulation(deck, sort_every=4) as sim:
            e, i, ids, tags = _plasma(sim)
        sr = StripRank(deck, rank, world, ghost=4, sort_every=4)
        try:
            sr.strip.load(ELECTRONS, *e, ids=ids, tags=tags)
            sr.strip.load(IONS, *i, ids=ids, tags=tags)
            sr.step(STEPS)
            out[rank] = ([sr.strip.download(s) for s in (ELECTRONS, IONS)], sr.field.field(FIELD_PHI))
        finally:
            sr.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_ranks_of_strips_equal_one_context(tmp_path):
    deck = small_deck(tmp_path, "periodic", collisions=False, bx=86.6, by=50.0)
    _, ref, phi_ref, _, _ = _reference(deck, 4, STEPS)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank_worker, args=(2, port, deck, out), nprocs=2, start_method="spawn", join=True)
    for s in range(2):
        both = {k: np.concatenate([out[0][0][s][k], out[1][0][s][k]]) for k in ref[s]}
        a, ia, _ = _rows(both)
        b, ib, _ = _rows(ref[s])
        assert np.array_equal(ia, ib) and np.array_equal(a, b)
    assert np.array_equal(out[0][1], phi_ref) and np.array_equal(out[1][1], phi_ref)
