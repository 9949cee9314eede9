"""Oracle known-answer tests for the source terms and BH orbits:
test/test_sinks.jl, test_nbody.jl, test_kepler_orbit.jl, test_self_gravity.jl,
test_fmr_gravity.jl (docs/phase7.md)."""
import json
import math
import os

import numpy as np
import pytest

NG = 3
DOC = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_documented.json")))


def _uniform(orc, n, rho, P, g):
    U = orc.state(n, n, n)
    U[0, NG:NG + n, NG:NG + n, NG:NG + n] = rho
    U[4, NG:NG + n, NG:NG + n, NG:NG + n] = P / (g - 1)
    return U


def _centres(n, dx, x0):
    return x0 + (np.arange(n) + 0.5) * dx


def test_sink_mass_accounting(orc):
    n, dx, g = 8, 0.1, 5 / 3
    U = _uniform(orc, n, 1.0, 1e-2, g)
    dU = np.zeros_like(U, order="F")
    bh = orc.make_bh((0.4, 0.4, 0.4), (0, 0, 0), 1.0, 1e-6, 1e6, 0.3)
    orc.add_sink_sources(dU, U, dx, dx, dx, [bh], 0.0, 0.0, 0.0, f_sink=1.0, torque_free=True)
    dV = dx ** 3
    dm_gas = -dU[0, NG:NG + n, NG:NG + n, NG:NG + n].sum() * dV
    rs, ts = orc.r_sink(bh), orc.t_sink(bh, 1.0)
    c = _centres(n, dx, 0.0)
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    r = np.sqrt((X - 0.4) ** 2 + (Y - 0.4) ** 2 + (Z - 0.4) ** 2)
    dm_bh = (U[0, NG:NG + n, NG:NG + n, NG:NG + n][r < rs] * dV / ts).sum()
    assert dm_gas == pytest.approx(dm_bh, abs=1e-14 * dm_bh)


def test_sink_torque_free_zero_torque(orc):
    n, dx, g = 8, 0.1, 5 / 3
    U = orc.state(n, n, n)
    c = _centres(n, dx, 0.0)
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    vx, vy = -Y, X
    a = (slice(NG, NG + n),) * 3
    U[(0,) + a] = 1.0
    U[(1,) + a] = vx
    U[(2,) + a] = vy
    U[(4,) + a] = 1e-2 / (g - 1) + 0.5 * (vx ** 2 + vy ** 2)
    dU = np.zeros_like(U, order="F")
    bh = orc.make_bh((0.4, 0.4, 0.4), (0, 0, 0), 1.0, 1e-6, 1e6, 0.3)
    orc.add_sink_sources(dU, U, dx, dx, dx, [bh], 0.0, 0.0, 0.0, torque_free=True)
    ddx, ddy, ddz = X - 0.4, Y - 0.4, Z - 0.4
    inside = np.sqrt(ddx ** 2 + ddy ** 2 + ddz ** 2) < orc.r_sink(bh)
    d2, d3, d4 = dU[(1,) + a], dU[(2,) + a], dU[(3,) + a]
    tq = np.maximum.reduce([np.abs(ddy * d4 - ddz * d3), np.abs(ddz * d2 - ddx * d4), np.abs(ddx * d3 - ddy * d2)])
    assert tq[inside].max() < 1e-14


def test_accrete_mass(orc):
    n, dx, g, dt = 8, 0.1, 5 / 3, 0.01
    U = _uniform(orc, n, 1.5, 1e-2, g)
    bh = orc.make_bh((0.4, 0.4, 0.4), (0, 0, 0), 1.0, 1e-6, 1e6, 0.25)
    rs = orc.r_sink(bh)
    c = _centres(n, dx, 0.0)
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    r = np.sqrt((X - 0.4) ** 2 + (Y - 0.4) ** 2 + (Z - 0.4) ** 2)
    M_before = (U[0, NG:NG + n, NG:NG + n, NG:NG + n][r < rs]).sum() * dx ** 3
    ts = orc.t_sink(bh)
    orc.accrete(bh, U, dx, dx, dx, 0.0, 0.0, 0.0, dt)
    assert bh.mass - 1.0 == pytest.approx(M_before / ts * dt, rel=1e-14)


def test_sink_density_threshold(orc):
    n, dx, g, dt = 8, 0.1, 5 / 3, 0.01
    U = _uniform(orc, n, 1e-3, 1e-2, g)
    ic = NG + n // 2
    U[0, ic, ic, ic] = 1.0
    bh = orc.make_bh((0.4, 0.4, 0.4), (0, 0, 0), 1.0, 1e-6, 1e6, 0.3)
    dU = np.zeros_like(U, order="F")
    orc.add_sink_sources(dU, U, dx, dx, dx, [bh], 0.0, 0.0, 0.0, torque_free=True, rho_sink_min=2e-3)
    dV = dx ** 3
    ts = orc.t_sink(bh)
    rate = -dU[0, NG:NG + n, NG:NG + n, NG:NG + n].sum() * dV
    assert rate == pytest.approx(1.0 * dV / ts, rel=1e-14)
    m0 = bh.mass
    orc.accrete(bh, U, dx, dx, dx, 0.0, 0.0, 0.0, dt, rho_sink_min=2e-3)
    dM = bh.mass - m0
    assert dM == pytest.approx(dV / ts * dt, rel=1e-10)
    bh2 = orc.make_bh((0.4, 0.4, 0.4), (0, 0, 0), 1.0, 1e-6, 1e6, 0.3)
    orc.accrete(bh2, U, dx, dx, dx, 0.0, 0.0, 0.0, dt)
    assert bh2.mass - 1.0 > dM


def _pair(orc, eps=1e-4):
    return orc.bh_array([orc.make_bh((0.5, 0, 0), (0, 0.5, 0), 0.5, eps, 1e6, 0.01),
                         orc.make_bh((-0.5, 0, 0), (0, -0.5, 0), 0.5, eps, 1e6, 0.01)])


def test_nbody_kepler_ten_orbits(orc):
    bhs = _pair(orc)

    def energy(b):
        ke = sum(0.5 * b[i].mass * sum(v * v for v in b[i].vel) for i in range(2))
        d = [b[0].pos[t] - b[1].pos[t] for t in range(3)]
        return ke - b[0].mass * b[1].mass / math.sqrt(sum(x * x for x in d) + b[0].eps ** 2)

    def Lz(b):
        return sum(b[i].mass * (b[i].pos[0] * b[i].vel[1] - b[i].pos[1] * b[i].vel[0]) for i in range(2))

    E0, L0 = energy(bhs), Lz(bhs)
    T = 2 * math.pi
    dt = T / 500
    t, tend = 0.0, 10 * T
    F = np.zeros((2, 3))
    while t < tend:
        s = min(dt, tend - t)
        orc.nbody_step(bhs, 2, s, F)
        t += s
    assert abs(energy(bhs) - E0) / abs(E0) < 1e-3
    assert abs(Lz(bhs) - L0) / abs(L0) < 1e-3


def test_kepler_closure_and_agreement(orc):
    bhs = _pair(orc)
    p0 = [list(bhs[i].pos) for i in range(2)]
    st = orc.kepler_init(bhs)
    assert st[3] == pytest.approx(1.0, abs=1e-12) and st[6] == pytest.approx(1.0, abs=1e-12)
    orc.kepler_update(bhs, st, 2 * math.pi / st[3])
    for i in range(2):
        assert max(abs(bhs[i].pos[t] - p0[i][t]) for t in range(3)) < 1e-12
    bk = _pair(orc)
    st = orc.kepler_init(bk)
    bn = _pair(orc)
    dt = 2 * math.pi / 2000
    F = np.zeros((2, 3))
    t = 0.0
    for _ in range(500):
        orc.nbody_step(bn, 2, dt, F)
        t += dt
    orc.kepler_update(bk, st, t)
    for i in range(2):
        assert max(abs(bk[i].pos[q] - bn[i].pos[q]) for q in range(3)) < 1e-5
        assert max(abs(bk[i].vel[q] - bn[i].vel[q]) for q in range(3)) < 1e-5


def _sphere(n, dx, R, r0=1.0):
    c = (np.arange(n) + 0.5) * dx - 0.5
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    return np.asfortranarray(np.where(np.sqrt(X ** 2 + Y ** 2 + Z ** 2) < R, r0, 0.0))


def _ratio_err(orc, N):
    dx = 1.0 / N
    phi = orc.solve_poisson_isolated(_sphere(N, dx, 0.15), dx, dx, dx)
    jc = round(0.5 / dx + 0.5)
    r = lambda i: math.sqrt(((i - 0.5) * dx - 0.5) ** 2 + 2 * ((jc - 0.5) * dx - 0.5) ** 2)
    iA, iB = round(0.75 / dx + 0.5), round(0.85 / dx + 0.5)
    num = phi[iA - 1, jc - 1, jc - 1] / phi[iB - 1, jc - 1, jc - 1]
    return abs(num - r(iB) / r(iA)) / (r(iB) / r(iA))


def test_poisson_ratio_convergence_and_self_energy(orc):
    doc = DOC["poisson_sphere"]
    e16, e32 = _ratio_err(orc, 16), _ratio_err(orc, 32)
    assert e32 < e16 and e32 < 0.01
    assert round(e32, 4) == doc["ratio_err_N32"] and round(e16, 3) == doc["ratio_err_N16"]
    N, dx = 32, 1 / 32
    rho = _sphere(N, dx, 0.15)
    M = rho.sum() * dx ** 3
    phi = orc.solve_poisson_isolated(rho, dx, dx, dx)
    err = abs((0.5 * (rho * phi).sum() * dx ** 3 + 3 * M ** 2 / (5 * 0.15)) / (3 * M ** 2 / (5 * 0.15)))
    assert err < 0.10 and round(err, 3) == doc["self_energy_err_N32"]


def test_fft_matches_numpy(orc):
    a = np.random.default_rng(0).standard_normal((8, 16, 4)) + 0j
    for shape in ((8, 16, 4), (6, 5, 3)):
        a = np.random.default_rng(1).standard_normal(shape)
        re = np.asfortranarray(a.copy())
        im = np.zeros_like(re, order="F")
        orc.lib().orc_fft3d(orc._p(re), orc._p(im), *shape, 0)
        ref = np.fft.fftn(a)
        assert np.abs(re + 1j * im - ref).max() <= 1e-13 * np.abs(ref).max()


def test_self_gravity_symmetric_zero_net_force(orc):
    n = 16
    dx = 1.0 / n
    U = orc.state(n, n, n)
    c = (np.arange(n) + 0.5) * dx - 0.5
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    rho = np.where(np.sqrt(X ** 2 + Y ** 2 + Z ** 2) < 0.25, 1.0, 1e-4)
    a = (slice(NG, NG + n),) * 3
    U[(0,) + a] = rho
    U[(4,) + a] = rho * 1e-3
    dU = np.zeros_like(U, order="F")
    orc.add_self_gravity_source(dU, U, dx, dx, dx)
    Fs = np.abs(dU[(slice(1, 4),) + a]).max() * dx ** 3
    for q in (1, 2, 3):
        assert abs(dU[(q,) + a].sum() * dx ** 3) < 0.01 * Fs * n ** 3


def _sg_grid(orc, nc=8, L=0.5, ratio=4, R=0.2, r0=1.0, rbg=1e-4, g=5 / 3, e=1e-3):
    dxc = 2 * L / nc
    Uc = orc.state(nc, nc, nc)
    c = (np.arange(nc) + 0.5) * dxc - L
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    rho = np.where(np.sqrt(X ** 2 + Y ** 2 + Z ** 2) < R, r0, rbg)
    a = (slice(NG, NG + nc),) * 3
    Uc[(0,) + a] = rho
    Uc[(4,) + a] = rho * e
    orc.fill_ghost_3d_outflow(Uc)
    lo, hi = nc // 4 + 1, 3 * (nc // 4)
    G = orc.FMRGrid(Uc, dxc, lo, hi, lo, hi, lo, hi, ratio, g, rho_floor=1e-12, P_floor=1e-12)
    dxf = dxc / ratio
    nf = (hi - lo + 1) * ratio
    xf0 = (lo - 1) * dxc - L
    cf = (np.arange(nf) + 0.5) * dxf + xf0
    X, Y, Z = np.meshgrid(cf, cf, cf, indexing="ij")
    rf = np.where(np.sqrt(X ** 2 + Y ** 2 + Z ** 2) < R, r0, rbg)
    af = (slice(NG, NG + nf),) * 3
    G.Uf[(0,) + af] = rf
    G.Uf[(4,) + af] = rf * e
    G.prolong_fine_ghosts()
    return G


def test_fmr_gravity_regression_and_poisson(orc):
    G1, G2 = _sg_grid(orc), _sg_grid(orc)
    G1.step(1e-4)
    G2.step(1e-4, self_gravity=False)
    assert np.array_equal(G1.Uc, G2.Uc) and np.array_equal(G1.Uf, G2.Uf)
    G = _sg_grid(orc)
    G.restrict_density_to_coarse()
    n = G.s.ncx
    rho = np.asfortranarray(G.Uc[0, NG:NG + n, NG:NG + n, NG:NG + n])
    phi_ref = orc.solve_poisson_isolated(rho, G.s.dxc, G.s.dxc, G.s.dxc)
    phic, phif = _sg_grid(orc).solve_poisson()
    assert np.array_equal(phic, phi_ref)
    assert phif.shape == (G.s.nfx,) * 3


def test_fmr_gravity_momentum_and_infall(orc):
    G = _sg_grid(orc)
    G.step(1e-4, self_gravity=True)
    nc, nf = G.s.ncx, G.s.nfx
    ac = (slice(NG, NG + nc),) * 3
    af = (slice(NG, NG + nf),) * 3
    Mc = G.Uc[(0,) + ac].sum()
    for q in (1, 2, 3):
        assert abs(G.Uc[(q,) + ac].sum()) / Mc < 1e-10
        assert abs(G.Uf[(q,) + af].sum()) / Mc < 1e-10
    G = _sg_grid(orc, rbg=1e-6, e=1e-4)
    G.step(5e-4, self_gravity=True)
    dxf = G.s.dxf
    xf0 = (G.s.ci_lo - 1) * G.s.dxc - 0.5
    cf = (np.arange(nf) + 0.5) * dxf + xf0
    X, Y, Z = np.meshgrid(cf, cf, cf, indexing="ij")
    r = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    rad = (G.Uf[(1,) + af] * X + G.Uf[(2,) + af] * Y + G.Uf[(3,) + af] * Z) / np.maximum(r, 1e-300)
    assert rad.sum() * dxf ** 3 < 0.0


def test_diagnostics_match_reference_formulas(orc):
    """The oracle's src/diagnostics.jl restatement against numpy evaluations
    of the reference's broadcast expressions (gas energy, kinetic energy,
    momentum, angular momentum about the origin, bound mass with the BH
    potential) on a random state with two BHs."""
    from binary_ic import binary_setup
    U, dx, x0, specs = binary_setup(orc, n=16)
    rng = np.random.default_rng(3)
    a = (slice(3, -3),) * 3
    for q in (1, 2, 3):
        U[(q,) + a] = rng.normal(0.0, 0.3, U[(q,) + a].shape) * U[(0,) + a]
    bhs = [orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"]) for s in specs]
    g = 4 / 3
    out = orc.diagnostics(U, dx, dx, dx, x0, x0, x0, bhs, g)
    n = 16
    c = x0 + (np.arange(1, n + 1) - 0.5) * dx
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    r, mx, my, mz, E = (U[(q,) + a] for q in range(5))
    rs = np.maximum(r, 1e-30)
    ke = 0.5 * (mx ** 2 + my ** 2 + mz ** 2) / rs
    P = np.maximum((g - 1) * (E - rs * ke), 0.0)
    phi = np.zeros_like(r)
    for s in specs:
        phi -= s["mass"] / np.sqrt((X - s["pos"][0]) ** 2 + (Y - s["pos"][1]) ** 2 + (Z - s["pos"][2]) ** 2
                                   + s["eps"] ** 2)
    bound = (ke + P / ((g - 1) * rs) + phi) <= 0
    dV = dx ** 3
    ref = [E.sum(), ke.sum(), mx.sum(), my.sum(), mz.sum(), (Y * mz - Z * my).sum(), (Z * mx - X * mz).sum(),
           (X * my - Y * mx).sum(), rs[bound].sum(), r.sum()]
    ref = np.array(ref) * dV
    scale = np.array([abs(E).sum(), ke.sum(), abs(mx).sum(), abs(my).sum(), abs(mz).sum()] +
                     [np.abs(X * my).sum() + np.abs(Y * mz).sum() + np.abs(Z * mx).sum()] * 3 +
                     [rs.sum(), r.sum()]) * dV
    assert 0 < bound.sum() < bound.size
    assert np.all(np.abs(out - ref) <= 1e-13 * scale), (out, ref)
