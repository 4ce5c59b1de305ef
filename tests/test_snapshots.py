"""Snapshot files in the reference's binary layouts (pic2d_Snapshots.f90): SAVE_GLOBAL_2D_ARRAY (:1207-1355),
SAVE_ALL_VDF1D (:1359-1544) and SAVE_ALL_VDF2D (:1548-1705), decoded here independently from the reference's record
arithmetic (offsets in 4-byte units), on synthetic arrays. Runs without a GPU."""
import numpy as np

from edipic_b200 import snapshots


def test_global_2d_array_layout(tmp_path):
    nx, ny, dx = 7, 5, 2.5e-5
    arr = np.arange(nx * ny, dtype=np.float32).reshape(ny, nx) * 0.5 - 3.0
    path = tmp_path / "_0003_F_V_2D.bin"
    snapshots.write_2d(path, arr, dx)
    raw = np.fromfile(path, dtype=np.float32)
    gmi = nx - 1
    assert raw.size == (gmi + 2) * (ny + 1)
    # row 0: REAL(global_maximal_i + 1), then REAL(i * delta_x_m)
    assert raw[0] == np.float32(gmi + 1)
    assert np.array_equal(raw[1:gmi + 2], np.array([np.float32(i * dx) for i in range(nx)]))
    for j in range(ny):
        shift = (gmi + 2) + j * (gmi + 2)   # shifthead of row j, one cluster
        assert raw[shift] == np.float32(j * dx)
        assert np.array_equal(raw[shift + 1:shift + 1 + nx], arr[j])
    x, y, back = snapshots.read_2d(path)
    assert np.array_equal(back, arr)


def _write_vdf(tmp_path, two_d):
    import ctypes as C

    from edipic_b200 import library
    lib = library()
    nbx, nby, nme, nve, nmi, nvi, ns = 3, 2, 2, 3, 1, 4, 2
    rle, rli, nb = 2 * nme * nve, 2 * nmi * nvi, nbx * nby
    rng = np.random.default_rng(0)
    e1 = rng.integers(0, 1000, (3, nb, rle)).astype(np.int32)
    i1 = rng.integers(0, 1000, (ns, 3, nb, rli)).astype(np.int32)
    e2 = rng.integers(0, 1000, (nb, rle, rle)).astype(np.int32)
    amu = np.array([39.948, 4.0026])
    i32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    p1, p2 = str(tmp_path / "_0001_vdf1d.bin"), str(tmp_path / "_0001_vdf2d.bin")
    assert lib.edp_write_vdf1d(p1.encode(), nbx, nby, 65.0, 48.0, 1e-5, nme, nve, nmi, nvi, ns, 2.5,
                               amu.ctypes.data_as(C.POINTER(C.c_double)), i32(e1), i32(i1)) == 0
    assert lib.edp_write_vdf2d(p2.encode(), nbx, nby, 65.0, 48.0, 1e-5, nme, nve, 2.5, i32(e2)) == 0
    return dict(nbx=nbx, nby=nby, rle=rle, rli=rli, ns=ns, e1=e1, i1=i1, e2=e2, amu=amu, p1=p1, p2=p2)


def test_vdf_files_layout(tmp_path):
    d = _write_vdf(tmp_path, True)
    raw = np.fromfile(d["p1"], dtype=np.int32)
    rawf = raw.view(np.float32)
    nbx, nby, rle, rli, ns = d["nbx"], d["nby"], d["rle"], d["rli"], d["ns"]
    assert list(raw[:9]) == [nbx, nby, -rle // 2, rle // 2 - 1, -rli // 2, rli // 2 - 1, 3, 4, ns]
    assert rawf[9] == np.float32(2.5) and np.array_equal(rawf[10:10 + ns], d["amu"].astype(np.float32))
    one = 4 + 3 * rle + ns * 3 * rli
    xs = [np.float32((0.0 + i * 65.0 / nbx) * 1e-5) for i in range(nbx)] + [np.float32(65.0 * 1e-5)]
    ys = [np.float32((0.0 + j * 48.0 / nby) * 1e-5) for j in range(nby)] + [np.float32(48.0 * 1e-5)]
    xs[0], ys[0] = np.float32(0.0), np.float32(0.0)
    for j in range(nby):
        for i in range(nbx):
            n = i + j * nbx
            s0 = 9 + 1 + ns + (j * nbx + i) * one
            assert list(rawf[s0:s0 + 4]) == [xs[i], xs[i + 1], ys[j], ys[j + 1]]
            rec = raw[s0 + 4:s0 + one]
            exp = np.concatenate([d["e1"][c, n] for c in range(3)] +
                                 [d["i1"][s, c, n] for s in range(ns) for c in range(3)])
            assert np.array_equal(rec, exp)
    assert raw.size == 9 + 1 + ns + nbx * nby * one
    raw2 = np.fromfile(d["p2"], dtype=np.int32)
    assert list(raw2[:5]) == [nbx, nby, -rle // 2, rle // 2 - 1, 3]
    one2 = 4 + rle * rle
    for n in range(nbx * nby):
        s0 = 5 + 1 + n * one2
        assert np.array_equal(raw2[s0 + 4:s0 + one2], d["e2"][n].ravel())
