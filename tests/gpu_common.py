"""Shared set-up of the GPU parity tests: synthetic decks, random particles and fields, oracle geometry."""
import numpy as np

import pyoracle
from edipic_b200 import PREC_MIXED, decks


def small_deck(tmp, kind, **kw):
    if kind == "periodic":
        return decks.write_deck(str(tmp), "cfg0", ncx=kw.pop("ncx", 64), ncy=kw.pop("ncy", 48), ppc=kw.pop("ppc", 16),
                                **kw)
    return decks.write_deck(str(tmp), "cfg2", ncx=kw.pop("ncx", 64), ncy=kw.pop("ncy", 64), ppc=kw.pop("ppc", 16),
                            inner=kw.pop("inner", (20, 24, 36, 32, -100.0)), **kw)


def oracle_geom(sim):
    p = sim.params
    inner = [(p.inner_ileft[k], p.inner_jbottom[k], p.inner_iright[k], p.inner_jtop[k]) for k in range(p.n_inner)]
    return pyoracle.geom(p.ncx, p.ncy, p.periodic_x, inner)


def random_particles(sim, n, seed=1, vscale=0.05, fast_fraction=0.05, precision=PREC_MIXED):
    """Uniform positions (snapped to the FP32 in-cell offsets the mixed layout stores), Maxwellian velocities plus
    a fraction of fast particles that cross cells and walls in one step."""
    p = sim.params
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, p.ncx, n)
    y = rng.uniform(0.0, p.ncy, n)
    if precision == PREC_MIXED:
        i, j = np.floor(x), np.floor(y)
        x = i + (x - i).astype(np.float32).astype(np.float64)
        y = j + (y - j).astype(np.float32).astype(np.float64)
    v = rng.normal(0.0, vscale, (3, n))
    fast = rng.random(n) < fast_fraction
    v[:, fast] *= 15.0
    if precision == PREC_MIXED:
        v = v.astype(np.float32).astype(np.float64)
    return x, y, v[0], v[1], v[2]


def random_field(sim, seed=2, amp=0.02, precision=PREC_MIXED):
    """A smooth random field on the reference node layout (periodic overlap columns consistent)."""
    p = sim.params
    rng = np.random.default_rng(seed)
    nyr, nxr = sim.ny_ref, sim.nx_ref
    jj, ii = np.meshgrid(np.arange(nyr), np.arange(nxr), indexing="ij")
    out = []
    for _ in range(2):
        f = np.zeros((nyr, nxr))
        for _m in range(4):
            kx = rng.integers(1, 4) * 2 * np.pi / p.ncx
            ky = rng.integers(1, 4) * np.pi / p.ncy
            f += amp * rng.normal() * np.cos(kx * ii + rng.uniform(0, 6.28)) * np.cos(ky * jj + rng.uniform(0, 6.28))
        if sim.periodic:
            f[:, p.ncx] = f[:, 0]
            f[:, p.ncx + 1] = f[:, 1]
        if precision == PREC_MIXED:
            f = f.astype(np.float32).astype(np.float64)
        out.append(f)
    return out


def match_by_id(a, b):
    """Row order of b matching the ids of a (both dicts of columns)."""
    ia = np.argsort(a["id"])
    ib = np.argsort(b["id"])
    assert np.array_equal(a["id"][ia], b["id"][ib])
    return ia, ib


def periodic_dx(d, period):
    return (d + 0.5 * period) % period - 0.5 * period


def contribution_bound(sim, x, y):
    """Per-node bound 2 * 2^-32 * (number of CIC contributions) * (wall factor) of the fixed-point deposit error,
    on the reference node layout."""
    p = sim.params
    cnt = np.zeros((sim.ny_ref, sim.nx_ref))
    i = np.minimum(np.floor(x).astype(int), p.ncx - 1 if not sim.periodic else p.ncx)
    j = np.minimum(np.floor(y).astype(int), p.ncy - 1)
    for di in (0, 1):
        for dj in (0, 1):
            np.add.at(cnt, (j + dj, i + di), 1.0)
    f = np.ones_like(cnt)
    if sim.periodic:
        n = p.ncx
        cnt[:, 1] += cnt[:, n + 1]
        cnt[:, n] += cnt[:, 0]
        cnt[:, 0] = cnt[:, n]
        cnt[:, n + 1] = cnt[:, 1]
        f[0, :] = f[-1, :] = 2.0
    else:
        f[0, :] = f[-1, :] = 2.0
        f[:, 0] = f[:, -1] = 2.0
        f[0, 0] = f[0, -1] = f[-1, 0] = f[-1, -1] = 4.0
    return 2.0 * 2.0 ** -32 * cnt * f + 1e-12
