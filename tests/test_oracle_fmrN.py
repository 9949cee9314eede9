"""The oracle's N-level FMR restatement (recursive fmr3d_step!, src/fmr3d.jl
:451-604, with ratio subcycles per level and ghosts from the parent at
alpha = s/r).  The reference has two levels; at N = 2 the restatement must
reproduce the two-level step bit for bit, and at N = 3 it must keep the
invariants the reference tests for two levels (test/test_fmr3d.jl:113-170:
conservation with Berger-Colella correction, a Sedov blast close to the
uniform fine-grid result)."""
import numpy as np
import pytest

NG = 3


def _sedov_levels(orc, nc=8, L=0.5, boxes=((3, 6, 3, 6, 3, 6, 2), (4, 5, 4, 5, 4, 5, 2)), g=5 / 3,
                  Pf=1e-5, rfl=1e-10, rbg=1.0):
    dxc = 2 * L / nc
    Uc = orc.state(nc, nc, nc)
    orc.sedov_ic_3d(Uc, dxc, dxc, dxc, g, E_blast=1.0, r_inject=0.15, rho_bg=rbg, P_floor=Pf,
                    x_offset=-L, y_offset=-L, z_offset=-L)
    orc.fill_ghost_3d_outflow(Uc)
    H = orc.FMRHierarchy(Uc, dxc, boxes, g, rho_floor=rfl, P_floor=Pf)
    # each level gets its own exact IC, its ghosts from the parent
    x0, dx = -L, dxc
    for k, (lo, hi, *_rest) in enumerate(boxes):
        r = boxes[k][6]
        x0 = x0 + (lo - 1) * dx
        dx = dx / r
        orc.sedov_ic_3d(H.levels[k + 1], dx, dx, dx, g, E_blast=1.0, r_inject=0.15, rho_bg=rbg,
                        P_floor=Pf, x_offset=x0, y_offset=x0, z_offset=x0)
        H.pairs[k].prolong_fine_ghosts()
    return H


def test_two_levels_reduce_to_fmr3d_step(orc):
    g = 5 / 3
    for sg in (False, True):
        H = _sedov_levels(orc, boxes=((3, 6, 3, 6, 3, 6, 4),))
        nc = 8
        Uc = H.levels[0].copy(order="F")
        G = orc.FMRGrid(Uc, 1 / 8, 3, 6, 3, 6, 3, 6, 4, g, rho_floor=1e-10, P_floor=1e-5, init=False)
        G.Uf[...] = H.levels[1]
        for _ in range(2):
            dt = H.cfl_dt(0.4)
            assert dt == G.cfl_dt(0.4)
            H.step(dt, self_gravity=sg, G_grav=0.7)
            G.step(dt, self_gravity=sg, G_grav=0.7)
        assert np.array_equal(H.levels[0], G.Uc) and np.array_equal(H.levels[1], G.Uf), sg


def test_three_level_cfl_is_min_over_levels(orc):
    H = _sedov_levels(orc)
    dts = [orc.cfl_dt_3d(U, dx, dx, dx, 5 / 3, 0.4) for U, dx in
           zip(H.levels, (1 / 8, 1 / 16, 1 / 32))]
    assert H.cfl_dt(0.4) == min(dts[0], 2 * dts[1], 4 * dts[2])


def test_three_level_sedov_conserves_and_tracks_uniform(orc):
    # the blast stays inside the domain: the base level conserves mass to
    # rounding through both Berger-Colella corrections
    H = _sedov_levels(orc, nc=16, boxes=((5, 12, 5, 12, 5, 12, 2), (5, 12, 5, 12, 5, 12, 2)))
    nc = 16
    a = (slice(NG, NG + nc),) * 3
    U0 = H.levels[0]
    # the first step replaces the covered coarse cells by the restriction of
    # the finer levels' own initial conditions: totals are taken after it
    t = H.cfl_dt(0.4)
    H.step(t)
    M0, E0 = U0[(0,) + a].sum(), U0[(4,) + a].sum()
    tend = 0.01
    while t < tend:
        dt = min(H.cfl_dt(0.4), tend - t)
        H.step(dt)
        t += dt
    assert abs(U0[(0,) + a].sum() - M0) / M0 < 1e-13
    # energy drifts by ~3e-7 with two levels as well (the reference allows 15 %)
    assert abs(U0[(4,) + a].sum() - E0) / E0 < 1e-5
    # the finest level against a uniform run at its resolution over its extent
    nf = 64
    dxf = 1.0 / nf
    Ur = orc.state(nf, nf, nf)
    orc.sedov_ic_3d(Ur, dxf, dxf, dxf, 5 / 3, E_blast=1.0, r_inject=0.15, rho_bg=1.0, P_floor=1e-5,
                    x_offset=-0.5, y_offset=-0.5, z_offset=-0.5)
    t = 0.0
    while t < tend:
        dt = min(orc.cfl_dt_3d(Ur, dxf, dxf, dxf, 5 / 3, 0.4), tend - t)
        orc.euler3d_step(Ur, dxf, dxf, dxf, dt, 5 / 3, rho_floor=1e-10, P_floor=1e-5)
        t += dt
    U2 = H.levels[2]
    n2 = 16
    i0 = 24  # the finest level starts at x = -0.125, cell 24 of the uniform grid
    rf = U2[0, NG:NG + n2, NG:NG + n2, NG:NG + n2]
    rr = Ur[0, NG + i0:NG + i0 + n2, NG + i0:NG + i0 + n2, NG + i0:NG + i0 + n2]
    assert np.abs(rf - rr).mean() / rr.mean() < 0.05  # the two-level bound of test_fmr3d.jl


def test_three_level_covered_cells_are_restrictions(orc):
    # after every step each covered parent cell holds the mean of its r^3
    # children (restriction runs after the children's subcycles; the flux
    # correction touches uncovered cells only)
    H = _sedov_levels(orc)
    for _ in range(3):
        H.step(H.cfl_dt(0.4))
    for k, (ilo, ihi, jlo, jhi, klo, khi, r) in enumerate(
            ((3, 6, 3, 6, 3, 6, 2), (4, 5, 4, 5, 4, 5, 2))):
        Up, Uc = H.levels[k], H.levels[k + 1]
        n = Uc.shape[1] - 2 * NG
        kids = Uc[:, NG:NG + n, NG:NG + n, NG:NG + n].reshape(5, n // r, r, n // r, r, n // r, r)
        mean = kids.mean(axis=(2, 4, 6))
        cov = Up[:, NG + ilo - 1:NG + ihi, NG + jlo - 1:NG + jhi, NG + klo - 1:NG + khi]
        assert np.allclose(cov, mean, rtol=1e-14, atol=0), k


def test_nested_coupled_step_without_bhs_is_the_nested_step(orc):
    from binary_ic import binary_nested_setup
    H1, *_ = binary_nested_setup(orc)
    H2, boxes, dx0, x0, _ = binary_nested_setup(orc)
    for t in (0.0, 1.0):
        dt = H1.cfl_dt(0.4)
        H1.step(dt, self_gravity=True)
        H2.coupled_step(orc.bh_array([]), 0, dt, t, x0, x0, x0, 1.0, True, True, 0.0, 0.0)
    for A, B in zip(H1.levels, H2.levels):
        assert np.array_equal(A, B)


def test_nested_coupled_step_sinks_and_orbit(orc):
    from binary_ic import binary_nested_setup
    H, boxes, dx0, x0, specs = binary_nested_setup(orc)
    bo = orc.bh_array([orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"])
                       for s in specs])
    a = (0,) + (slice(NG, -NG),) * 3
    t, M0, mb0 = 0.0, None, None
    for k in range(3):
        dt = H.cfl_dt(0.4)
        Fg = H.coupled_step(bo, 2, dt, t, x0, x0, x0, 1.0, True, True, 0.0, 2e-8)
        t += dt
        if k == 0:   # level 0 holds the restriction of the finer levels' own states from here on
            M0, mb0 = H.levels[0][a].sum() * dx0 ** 3, bo[0].mass + bo[1].mass
    assert np.isfinite(Fg).all() and np.abs(Fg).max() > 0
    # the sinks drained gas and the BHs gained it
    assert bo[0].mass + bo[1].mass > mb0 > 10.0
    assert H.levels[0][a].sum() * dx0 ** 3 < M0
    # the orbit moved the BHs (counter-clockwise, mirror-symmetric pair)
    assert bo[0].pos[1] > 0 and bo[1].pos[1] < 0
    assert abs(bo[0].pos[0] + bo[1].pos[0]) < 1e-3 * abs(bo[0].pos[0])
