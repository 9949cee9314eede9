"""Algorithmic floating-point operations of one SSP-RK3 step per active cell
(TEST INFRASTRUCTURE; prints the figures bench.py's FP-pipe fraction uses).

Runs the oracle's euler3d_step! (src/euler3d.jl:220-260) over the counting
scalar type of oracle/flops.cpp: every +, -, *, /, sqrt and comparison counts
one.  Workloads: the Sedov blast at t = 0.025 on 128^3 (the state the stage
kernels are profiled on; sedov_ic_3d!, gamma = 5/3, floors 1e-6) and the Sod
tube on 64^3 after 20 steps (gamma = 1.4, split at x = 0.5).

    python oracle/count_flops.py            # ~2-4 min on a few cores
"""
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import oracle as orc  # noqa: E402


def sedov(n=128, t_end=0.025):
    g, L = 5.0 / 3.0, 1.0
    dx = 2 * L / n
    U = orc.state(n, n, n)
    orc.sedov_ic_3d(U, dx, dx, dx, g, E_blast=1.0, r_inject=3.5 * dx, rho_bg=1.0, P_floor=1e-5,
                    x_offset=-L, y_offset=-L, z_offset=-L)
    kw = dict(rho_floor=1e-6, P_floor=1e-6)
    t = 0.0
    while t < t_end:
        dt = min(orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4), t_end - t)
        orc.euler3d_step(U, dx, dx, dx, dt, g, **kw)
        t += dt
    dt = orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4)
    return U, dx, dt, g, kw


def sod(n=64, steps=20):
    g, dx = 1.4, 1.0 / n
    U = orc.state(n, n, n)
    x = (np.arange(n) + 0.5) * dx
    left = (x < 0.5)[:, None, None]
    a = (slice(3, -3),) * 3
    U[(0,) + a] = np.where(left, 1.0, 0.125)
    U[(4,) + a] = np.where(left, 1.0, 0.1) / (g - 1)
    orc.fill_ghost_3d_outflow(U)
    kw = dict(rho_floor=1e-10, P_floor=1e-10)
    for _ in range(steps):
        orc.euler3d_step(U, dx, dx, dx, orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4), g, **kw)
    return U, dx, orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4), g, kw


def per_cell(name, make):
    U, dx, dt, g, kw = make()
    n = np.prod(orc.dims(U))
    t0 = time.time()
    c = orc.count_step_flops(U, dx, dx, dx, dt, g, **kw)
    return name, {k: v / n for k, v in c.items()}, time.time() - t0


if __name__ == "__main__":
    out = {}
    for name, make in (("sedov128_t0.025", sedov), ("sod64_step20", sod)):
        k, v, el = per_cell(name, make)
        out[k] = {key: round(float(val), 1) for key, val in v.items()}
        print(f"{k}: {out[k]} ({el:.0f} s)", file=sys.stderr)
    print(json.dumps(out))
