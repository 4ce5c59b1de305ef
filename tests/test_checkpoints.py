"""Checkpoint files in the reference's layouts (pic2d_Checkpoints.f90): the POSIX per-rank stream files (:702-1124)
and the MPI-IO ordered single file (:5-660), decoded here from the reference's write order and round-tripped through
the readers; the WELL19937a state of well_random_seed against the oracle's seeding, which is pinned to the
reference's own generator. Runs without a GPU."""
import ctypes as C

import numpy as np
import pytest

import pyoracle
from edipic_b200 import checkpoints as ck


def ranks(n_spec=1, counts=((5, 3), (0, 4), (7, 0))):
    rng = np.random.default_rng(1)
    out = []
    for r, (ne, ni) in enumerate(counts):
        h = rng.integers(-2 ** 31, 2 ** 31 - 1, ck.header_length(n_spec)).astype(np.int32)
        h[ck.H_TCNTR] = 1234
        h[ck.H_NE] = ne
        for s in range(n_spec):
            h[637 + 2 * s] = ni
        h[-1] = 0

        def rec(n):
            a = np.zeros(n, ck.REC)
            for f in ("x", "y", "vx", "vy", "vz"):
                a[f] = rng.normal(size=n)
            a["tag"] = rng.integers(0, 9, n)
            return a
        out.append(ck.Rank(h, np.zeros(0), rec(ne), [rec(ni) for _ in range(n_spec)]))
    return out


def test_posix_layout_and_round_trip(tmp_path):
    rk = ranks()
    paths = ck.write_posix(str(tmp_path), 1234, rk)
    assert paths[2].endswith("checkdir_00001234/Tcntr_00001234_proc_002.check")
    for r, path in enumerate(paths):
        raw = open(path, "rb").read()
        L = ck.header_length(1)
        assert np.array_equal(np.frombuffer(raw, np.int32, L), rk[r].header)
        # WRITE (19) of X, Y, VX, VY, VZ, tag per particle: 44-byte records after the header
        ne = int(rk[r].header[ck.H_NE])
        for k in range(ne):
            off = 4 * L + 44 * k
            x, y, vx, vy, vz = np.frombuffer(raw, np.float64, 5, off)
            tag = np.frombuffer(raw, np.int32, 1, off + 40)[0]
            assert (x, vz, tag) == (rk[r].electrons["x"][k], rk[r].electrons["vz"][k], rk[r].electrons["tag"][k])
        assert len(raw) == 4 * L + 44 * (ne + len(rk[r].ions[0]))
    back = ck.read_posix(str(tmp_path), 1234, 1)
    assert len(back) == 3
    for a, b in zip(rk, back):
        assert np.array_equal(a.header, b.header)
        assert np.array_equal(a.electrons, b.electrons) and np.array_equal(a.ions[0], b.ions[0])


@pytest.mark.parametrize("n_spec", [1, 2])
def test_mpiio_layout_and_round_trip(tmp_path, n_spec):
    rk = ranks(n_spec)
    path = ck.write_mpiio(str(tmp_path / "Tcntr_00001234.check"), rk)
    raw = open(path, "rb").read()
    L = ck.header_length(n_spec)
    # MPI_FILE_WRITE_ORDERED blocks: headers of all ranks, surface charges, electron rows, electron tags, ...
    for r in range(3):
        assert np.array_equal(np.frombuffer(raw, np.int32, L, 4 * L * r), rk[r].header)
    pos = 4 * L * 3
    rows = np.frombuffer(raw, np.float64, 5 * 12, pos).reshape(12, 5)
    el = np.concatenate([r.electrons for r in rk])
    assert np.array_equal(rows[:, 0], el["x"]) and np.array_equal(rows[:, 4], el["vz"])
    assert np.array_equal(np.frombuffer(raw, np.int32, 12, pos + 40 * 12), el["tag"])
    back = ck.read_mpiio(path, n_spec)
    assert len(back) == 3
    for a, b in zip(rk, back):
        assert np.array_equal(a.header, b.header)
        assert np.array_equal(a.electrons, b.electrons)
        for s in range(n_spec):
            assert np.array_equal(a.ions[s], b.ions[s])


def test_well_seed_state_matches_oracle():
    for seed in (1, 12345, 2 ** 31 - 1, 7):
        st, ind, func = ck.well_seed_state(seed)
        w = pyoracle.Well()
        pyoracle.lib().oracle_well_seed(C.byref(w), seed)
        assert np.array_equal(st.view(np.uint32), np.frombuffer(w.v, np.uint32))
        assert (ind, func) == (0, 1) and w.i == 0
