"""Seeded synthetic inputs with the shapes of the binary-BH supernova workload
(config: n=3 polytrope star M=10, R=1, G=1 at the origin; two m=5 BH sinks on
a circular orbit of separation 3 in the z=0 plane; sink radius 4 cells;
thermal bomb), built with the oracle's restatement of the reference's IC
generators (src/stellar_ic.jl), at sizes the oracle finishes in seconds."""
import math

import numpy as np

NG = 3


def binary_setup(orc, n=32, L=4.0, r_bomb=0.5, gamma=4.0 / 3.0, rho_floor=1e-8, P_floor=1e-10):
    dx = 2 * L / n
    U = orc.state(n, n, n)
    orc.polytrope_ic_3d(U, dx, dx, dx, gamma, 10.0, 1.0, x0=-L, y0=-L, z0=-L, rho_floor=rho_floor, P_floor=P_floor)
    orc.thermal_bomb(U, dx, dx, dx, 1.0, r_bomb, x0=-L, y0=-L, z0=-L)
    v = math.sqrt(10.0 / 3.0) / 2.0
    bhs = [dict(pos=(1.5, 0.0, 0.0), vel=(0.0, v, 0.0)), dict(pos=(-1.5, 0.0, 0.0), vel=(0.0, -v, 0.0))]
    for b in bhs:
        b.update(mass=5.0, eps=2 * dx, c_code=1e6, r_floor=4 * dx)
    return U, dx, -L, bhs


def binary_nested_setup(orc, n=16, L=4.0, sep=1.0, r_bomb=0.5, gamma=4.0 / 3.0, rho_floor=1e-8, P_floor=1e-10,
                        sink_cells=3):
    """Three nested levels of n^3 (ratio 2, each covering the middle half of
    its parent: [-L,L]^3, [-L/2,L/2]^3, [-L/4,L/4]^3), each with its own
    polytrope + thermal bomb initial state at its resolution and ghosts from
    its parent; two m=5 BHs at (+-sep/2, 0, 0) with sink radius `sink_cells`
    and softening 2 finest cells.  A level none of whose cell centres lies
    within r_bomb gets no bomb (thermal_bomb! would find no gas there; the
    covered centre of that level takes the finer levels' restriction).  Returns (hierarchy,
    dx0, x0, bh specs)."""
    dx0 = 2 * L / n
    lo, hi = n // 4 + 1, 3 * n // 4
    boxes = ((lo, hi, lo, hi, lo, hi, 2),) * 2
    U0 = orc.state(n, n, n)

    def fill(U, dx, x0):
        orc.polytrope_ic_3d(U, dx, dx, dx, gamma, 10.0, 1.0, x0=x0, y0=x0, z0=x0, rho_floor=rho_floor,
                            P_floor=P_floor)
        if math.sqrt(3.0) * dx / 2 < r_bomb:   # the cell centres nearest the origin
            orc.thermal_bomb(U, dx, dx, dx, 1.0, r_bomb, x0=x0, y0=x0, z0=x0)

    fill(U0, dx0, -L)
    orc.fill_ghost_3d_outflow(U0)
    H = orc.FMRHierarchy(U0, dx0, boxes, gamma, rho_floor=rho_floor, P_floor=P_floor)
    x0, dx = -L, dx0
    for k in range(2):
        x0 = x0 + (lo - 1) * dx
        dx = dx / 2
        fill(H.levels[k + 1], dx, x0)
        H.pairs[k].prolong_fine_ghosts()
    v = math.sqrt(10.0 / sep) / 2.0
    bhs = [dict(pos=(sep / 2, 0.0, 0.0), vel=(0.0, v, 0.0)), dict(pos=(-sep / 2, 0.0, 0.0), vel=(0.0, -v, 0.0))]
    for b in bhs:
        b.update(mass=5.0, eps=2 * dx, c_code=1e6, r_floor=sink_cells * dx)
    return H, boxes, dx0, -L, bhs
