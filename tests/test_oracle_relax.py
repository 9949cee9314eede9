"""The oracle's restatement of the Roche relaxation (src/relax_ic.jl) against
the reference's own tests (test/test_relax_ic.jl): source values, KE
convergence, thermal-energy accounting, and the co-rotating relaxation that
keeps the star at its orbital position."""
import numpy as np

NG = 3


def _polytrope(orc, nx=16, gamma=5 / 3, R_star=0.4, L=1.0):
    dx = 2 * L / nx
    U = orc.state(nx, nx, nx)
    orc.polytrope_ic_3d(U, dx, dx, dx, gamma, 0.5, R_star, x0=-L, y0=-L, z0=-L)
    return U, dx


def _totals(orc, U, dx):
    t = orc.diagnostics(U, dx, dx, dx, 0.0, 0.0, 0.0, [], 5 / 3)
    return t[0], t[1]


def _perturb(U, nx=16):
    a = (slice(NG, NG + nx),) * 3
    U[(1,) + a] += 0.05 * U[(0,) + a]


def test_damping_source_values(orc):
    # test/test_relax_ic.jl:163-189
    U, dU = orc.state(8, 8, 8), orc.state(8, 8, 8)
    a = (slice(NG, NG + 8),) * 3
    U[(0,) + a] = 1.0
    U[(1,) + a] = 1.0
    U[(4,) + a] = 2.5
    orc.relax_damping_source(dU, U, 0.1, 0.1, 0.1, 0.0, 0.0, 0.0, 0.5)
    c = (NG, NG, NG)
    assert abs(dU[(1,) + c] + 2.0) <= 2e-12 and abs(dU[(4,) + c] + 2.0) <= 2e-12
    assert dU[(2,) + c] == 0.0 and dU[(3,) + c] == 0.0


def test_rotating_frame_source_values(orc):
    # test/test_relax_ic.jl:242-267
    U, dU = orc.state(8, 8, 8), orc.state(8, 8, 8)
    a = (slice(NG, NG + 8),) * 3
    U[(0,) + a] = 2.0
    U[(1,) + a] = 2.0
    U[(4,) + a] = 5.0
    orc.rotating_frame_source(dU, U, 0.1, 0.1, 0.1, 0.0, 0.0, 0.0, 0.5)
    c = (NG, NG, NG)
    assert np.isclose(dU[(1,) + c], 0.025, rtol=1e-12, atol=0)
    assert np.isclose(dU[(2,) + c], -1.975, rtol=1e-12, atol=0)
    assert np.isclose(dU[(4,) + c], 0.025, rtol=1e-12, atol=0)
    assert abs(dU[(3,) + c]) <= 1e-14


def test_relax_converges_and_keeps_thermal_energy(orc):
    # test/test_relax_ic.jl:41-58 and :102-127
    U, dx = _polytrope(orc)
    E0, KE0 = _totals(orc, U, dx)
    _perturb(U)
    t, n, kr = orc.relax_ic(U, dx, dx, dx, 5 / 3, t_damp=0.1, t_max=0.5, rho_floor=1e-10, P_floor=1e-10,
                            KE_tol=0.01)
    assert kr < 0.01 and n > 0 and t > 0.0
    E1, KE1 = _totals(orc, U, dx)
    assert E1 - KE1 >= 0.99 * (E0 - KE0)


def test_relax_with_bh_converges(orc):
    # test/test_relax_ic.jl:132-158: a BH beside the star, still < 5 %
    U, dx = _polytrope(orc)
    _perturb(U)
    bh = orc.make_bh((0.8, 0.0, 0.0), (0.0, 0.0, 0.0), 0.1, 0.1, 1e6, 0.05)
    t, n, kr = orc.relax_ic(U, dx, dx, dx, 5 / 3, bhs=[bh], x0=-1.0, y0=-1.0, z0=-1.0, t_damp=0.1, t_max=0.5,
                            rho_floor=1e-10, P_floor=1e-10, KE_tol=0.05)
    assert kr < 0.05 and n > 0


def test_corotating_relaxation_holds_the_star(orc):
    # test/test_relax_ic.jl:194-237
    nx, L = 16, 1.0
    dx = 2 * L / nx
    Ms, Mb, a = 0.5, 0.5, 1.0
    x_star, x_bh = -Mb * a / (Ms + Mb), Ms * a / (Ms + Mb)
    Om = np.sqrt((Ms + Mb) / a ** 3)
    U = orc.state(nx, nx, nx)
    orc.polytrope_ic_3d(U, dx, dx, dx, 5 / 3, Ms, 0.3, x0=-L, y0=-L, z0=-L, x_center=x_star)
    bh = orc.make_bh((x_bh, 0.0, 0.0), (0.0, 0.0, 0.0), Mb, 0.05, 20.0, 0.02)
    c = -L + (np.arange(nx) + 0.5) * dx

    def com_x(V):
        rho = V[0, NG:NG + nx, NG:NG + nx, NG:NG + nx]
        return float((rho * c[:, None, None]).sum() / rho.sum())

    com0 = com_x(U)
    t, n, kr = orc.relax_ic(U, dx, dx, dx, 5 / 3, bhs=[bh], x0=-L, y0=-L, z0=-L, t_damp=0.1, t_max=1.0,
                            KE_tol=0.0, Omega=Om, self_gravity=True)
    assert n > 5 and np.isfinite(U).all() and np.isfinite(kr)
    assert abs(com_x(U) - com0) < 0.15 * a
