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
