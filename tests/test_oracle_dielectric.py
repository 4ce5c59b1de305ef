"""The oracle's dielectric inner objects (the ε-weighted operator of SolverInitialization and the outline charge of
DO_*_COLL_WITH_INNER_OBJECT) against properties of the reference's algorithm: ε = 1 gives the vacuum solution; a very
large ε makes the object an equipotential; symmetric data give a symmetric potential; an absorbed particle puts exactly
its charge on two neighbouring outline nodes next to the crossing, on the side it crossed."""
import numpy as np

import pyoracle

NC = 32
OBJ = (12, 10, 20, 22)


def geom():
    return pyoracle.geom(NC, NC, False, [OBJ])


def test_unit_permittivity_is_vacuum():
    g = geom()
    rng = np.random.default_rng(0)
    rho = rng.normal(size=pyoracle.nodes_shape(g))
    walls = [0.0, 1.0, 0.0, 0.0]
    a, _, _ = pyoracle.cg_solve_eps(g, rho, walls, [0.0], [1.0])
    b, _, _ = pyoracle.cg_solve_eps(pyoracle.geom(NC, NC, False), rho, walls, [], [])
    assert np.abs(a - b).max() < 1e-9


def test_large_permittivity_equipotential_and_symmetry():
    g = geom()
    rho = np.zeros(pyoracle.nodes_shape(g))
    walls = [0.0, 1.0, 0.5, 0.5]
    phi, _, _ = pyoracle.cg_solve_eps(g, rho, walls, [0.0], [1.0e6])
    il, jb, ir, jt = OBJ
    inside = phi[jb:jt + 1, il:ir + 1]
    assert inside.max() - inside.min() < 1e-4
    # left/right symmetric walls and an object centred in x: phi(i) = phi(N - i)
    g2 = pyoracle.geom(NC, NC, False, [(10, 8, 22, 20)])
    phi2, _, _ = pyoracle.cg_solve_eps(g2, rho, walls, [0.0], [4.0])
    assert np.abs(phi2 - phi2[:, ::-1]).max() < 1e-9


def test_outline_charge():
    g = geom()
    il, jb, ir, jt = OBJ
    cases = [  # (x, y, vx, vy): crossing the left, top, right and bottom sides
        (il + 0.3, 15.25, 0.5, 0.0, [(il, 15), (il, 16)], [0.75, 0.25]),
        (14.6, jt - 0.2, 0.0, -0.5, [(14, jt), (15, jt)], [0.4, 0.6]),
        (ir - 0.1, 13.7, -0.4, 0.0, [(ir, 14), (ir, 13)], [0.7, 0.3]),
        (18.2, jb + 0.1, 0.0, 0.3, [(19, jb), (18, jb)], [0.2, 0.8]),
    ]
    for x, y, vx, vy, nodes, frac in cases:
        surf = np.zeros(pyoracle.nodes_shape(g))
        assert pyoracle.inner_hit(g, [3.0], x, y, vx, vy, 1.0, -1.0, surf) == 0
        assert abs(surf.sum() + 1.0) < 1e-12
        for (i, j), f in zip(nodes, frac):
            assert abs(surf[j, i] + f) < 1e-12, ((i, j), surf[j, i], f)
    surf = np.zeros(pyoracle.nodes_shape(g))   # a metal object takes no outline charge
    assert pyoracle.inner_hit(g, [0.0], il + 0.3, 15.25, 0.5, 0.0, 1.0, -1.0, surf) == 0 and not surf.any()
