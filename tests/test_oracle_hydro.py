"""Oracle pins against the reference's hydro tests and documented accuracy:
Sod (test/test_sod3d.jl, docs/phase1.md:36-43), Sedov (test/test_sedov.jl,
docs/phase1.md:50-58) and FMR (test/test_fmr3d.jl, docs/phase2.md:56-61)."""
import json
import math
import os

import numpy as np

from analytic import sod_errors

NG = 3
DOC = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_documented.json")))


def _run_sod(orc, d):
    U, dims, (dx, dy, dz) = orc.sod_ic_3d(d)
    t = 0.0
    while t < 0.2:
        dt = min(orc.cfl_dt_3d(U, dx, dy, dz, 1.4, 0.4), 0.2 - t)
        orc.euler3d_step(U, dx, dy, dz, dt, 1.4)
        t += dt
    return sod_errors(U, d, dims, (dx, dy, dz)["xyz".index(d)], 0.2)


def test_sod_matches_documented_L1_and_symmetry(orc):
    e = {d: _run_sod(orc, d) for d in "xyz"}
    doc = DOC["sod_L1_128x4x4"]
    for d in "xyz":
        assert all(x < 5e-2 for x in e[d])
        assert round(e[d][0], 4) == doc["rho"]
        assert round(e[d][1], 4) == doc["v"]
        assert round(e[d][2], 4) == doc["p"]
    assert abs(e["x"][0] - e["y"][0]) / e["x"][0] < 1e-10
    assert abs(e["x"][0] - e["z"][0]) / e["x"][0] < 1e-10


def test_sedov_radius_energy_symmetry(orc):
    g, n, L = 5 / 3, 32, 1.0
    dx = 2 * L / n
    U = orc.state(n, n, n)
    orc.sedov_ic_3d(U, dx, dx, dx, g, E_blast=1.0, rho_bg=1.0, P_floor=1e-5, x_offset=-L, y_offset=-L, z_offset=-L)
    act = (4, slice(NG, NG + n), slice(NG, NG + n), slice(NG, NG + n))
    E0 = U[act].sum() * dx ** 3
    t = 0.0
    while t < 0.1:
        dt = min(orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4), 0.1 - t)
        orc.euler3d_step(U, dx, dx, dx, dt, g, rho_floor=1e-6, P_floor=1e-6)
        t += dt
    E1 = U[act].sum() * dx ** 3
    assert abs(E1 - E0) / E0 < 0.05
    rho = U[0, NG:NG + n, NG:NG + n, NG:NG + n]
    c = -L + (np.arange(n) + 0.5) * dx
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    R_num = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)[rho > 1.5].max()
    R_exact = (1.0 / 0.4942) ** 0.2 * 0.1 ** 0.4
    err = abs(R_num - R_exact) / R_exact
    assert err < 0.10
    assert round(R_num, 3) == DOC["sedov_32"]["R_num"]
    mid = NG + n // 2
    rx = U[0, NG:NG + n, mid, mid]
    ry = U[0, mid, NG:NG + n, mid]
    rz = U[0, mid, mid, NG:NG + n]
    h = n // 2 - 1
    assert np.abs(rx[h:] - ry[h:]).max() / rx.max() < 0.1
    assert np.abs(rx[h:] - rz[h:]).max() / rx.max() < 0.1


def test_fmr_sedov_vs_uniform(orc):
    g, Eb, rbg, Pf, rfl, rinj, cfl, tend = 5 / 3, 1.0, 1.0, 1e-5, 1e-10, 0.15, 0.4, 0.01
    nc, L, ratio = 8, 0.5, 4
    dxc = 2 * L / nc
    dxf = dxc / ratio
    lo, hi = 3, 6
    nf = (hi - lo + 1) * ratio
    xlo = -L
    xflo = (lo - 1) * dxc + xlo
    Uc = orc.state(nc, nc, nc)
    orc.sedov_ic_3d(Uc, dxc, dxc, dxc, g, E_blast=Eb, r_inject=rinj, rho_bg=rbg, P_floor=Pf,
                    x_offset=xlo, y_offset=xlo, z_offset=xlo)
    orc.fill_ghost_3d_outflow(Uc)
    G = orc.FMRGrid(Uc, dxc, lo, hi, lo, hi, lo, hi, ratio, g, rho_floor=rfl, P_floor=Pf)
    orc.sedov_ic_3d(G.Uf, dxf, dxf, dxf, g, E_blast=Eb, r_inject=rinj, rho_bg=rbg, P_floor=Pf,
                    x_offset=xflo, y_offset=xflo, z_offset=xflo)
    G.prolong_fine_ghosts()
    act = (4, slice(NG, NG + nc), slice(NG, NG + nc), slice(NG, NG + nc))
    E0 = Uc[act].sum() * dxc ** 3
    t = 0.0
    while t < tend:
        dt = min(G.cfl_dt(cfl), tend - t)
        G.step(dt)
        t += dt
    E1 = Uc[act].sum() * dxc ** 3
    nr = nc * ratio
    Ur = orc.state(nr, nr, nr)
    orc.sedov_ic_3d(Ur, dxf, dxf, dxf, g, E_blast=Eb, r_inject=rinj, rho_bg=rbg, P_floor=Pf,
                    x_offset=xlo, y_offset=xlo, z_offset=xlo)
    t = 0.0
    while t < tend:
        dt = min(orc.cfl_dt_3d(Ur, dxf, dxf, dxf, g, cfl), tend - t)
        orc.euler3d_step(Ur, dxf, dxf, dxf, dt, g, rho_floor=rfl, P_floor=Pf)
        t += dt
    i0 = round((xflo - xlo) / dxf)
    s = slice(NG + i0, NG + i0 + nf)
    rf = G.Uf[0, NG:NG + nf, NG:NG + nf, NG:NG + nf]
    rr = Ur[0, s, s, s]
    L1 = np.mean(np.abs(rf - rr)) / np.mean(rr)
    assert np.isfinite(G.Uc).all() and np.isfinite(G.Uf).all()
    assert abs(E1 - E0) / E0 < 0.15
    assert L1 < 0.05
    assert round(L1, 4) == DOC["fmr_sedov"]["L1_rel"]
