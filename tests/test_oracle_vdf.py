"""The oracle's VDF binning (oracle_vdf, restating CALCULATE_ELECTRON_VDF, pic2d_VelocityDistributions.f90:3-206)
against a direct numpy statement of the same rules on random particles: boxes split at i * xmax / nbx, bins
INT(v fvc) minus one for negative v, skipped particles, the 2D vx-vy layout."""
import numpy as np

import pyoracle


def numpy_vdf(x, y, v, nbox, xmax, ymax, fvc, nmv, nvb):
    nbx, nby = nbox
    vmin = -nmv * nvb
    rl = -2 * vmin
    h1 = np.zeros((3, nbx * nby, rl), np.int32)
    h2 = np.zeros((nbx * nby, rl, rl), np.int32)
    xs = [i * xmax / nbx for i in range(1, nbx)]
    ys = [j * ymax / nby for j in range(1, nby)]
    skip = 0
    for k in range(len(x)):
        ib = next((i for i, s in enumerate(xs) if x[k] < s), nbx - 1)
        jb = next((j for j, s in enumerate(ys) if y[k] < s), nby - 1)
        b = []
        for c in range(3):
            t = int(v[c][k] * fvc)          # truncation toward zero, as INT
            if v[c][k] < 0:
                t -= 1
            b.append(t)
        if any(t < vmin or t > -vmin - 1 for t in b):
            skip += 1
            continue
        n = ib + jb * nbx
        for c in range(3):
            h1[c, n, b[c] - vmin] += 1
        h2[n, b[1] - vmin, b[0] - vmin] += 1
    return h1, h2, skip


def test_oracle_vdf_matches_numpy():
    rng = np.random.default_rng(3)
    n = 4000
    x = rng.uniform(0, 64, n)
    y = rng.uniform(0, 48, n)
    v = rng.normal(0, 0.05, (3, n))
    v[:, :10] = [[-2.0 / 240], [0.0], [1.0 / 240]] * np.ones((3, 10))   # exact bin edges, negative and positive
    x[:5] = [64.0 / 3, 2 * 64.0 / 3, 0.0, 64.0, 63.999]
    ps = pyoracle.ParticleSet(x, y, v[0], v[1], v[2])
    for nbox, nmv, nvb in [((1, 1), 4, 10), ((3, 2), 3, 8), ((2, 5), 2, 3)]:
        fvc = 24.0 * nvb
        h1, h2, sk = pyoracle.vdf(ps, nbox, 64.0, 48.0, fvc, nmv, nvb, True)
        r1, r2, rs = numpy_vdf(x, y, v, nbox, 64.0, 48.0, fvc, nmv, nvb)
        assert np.array_equal(h1, r1)
        assert np.array_equal(h2, r2)
        assert sk == rs
        assert h1[0].sum() + sk == n
