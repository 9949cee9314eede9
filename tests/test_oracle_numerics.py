"""Oracle known-answer tests: WENO5 exactness, SSP-RK3 identity/order,
HLLC rotations, BlackHole sink radii (test/test_weno5.jl, test_rk3.jl,
test_blackhole.jl)."""
import math

import numpy as np
import pytest

NG = 3


def test_weno5_exact_linear_and_quadratic(orc):
    # test/test_weno5.jl:1-22
    xs = np.arange(-2.0, 4.0)
    v = xs.copy()
    vL = orc.weno5_left(*v[0:5])
    vR = orc.weno5_right(*v[1:6])
    assert abs(vL - 0.5) < 1e-13 and abs(vR - 0.5) < 1e-13
    v2 = xs ** 2 + 1.0 / 12.0
    assert abs(orc.weno5_left(*v2[0:5]) - 0.25) < 1e-13
    assert abs(orc.weno5_right(*v2[1:6]) - 0.25) < 1e-13


def test_rk3_zero_rhs_identity(orc):
    # test/test_rk3.jl:59-66 through the Euler stage combines: a uniform state
    # at rest has zero flux divergence, so one step leaves it unchanged.
    U = orc.state(6, 5, 4)
    U[0] = 1.3
    U[4] = 2.0
    U0 = U.copy(order="F")
    orc.euler3d_step(U, 0.1, 0.1, 0.1, 0.05, 1.4)
    act = (slice(None), slice(NG, -NG), slice(NG, -NG), slice(NG, -NG))
    np.testing.assert_allclose(U[act], U0[act], rtol=1e-14, atol=0)


def _rk3_generic(u, L, dt):
    # src/rk3.jl:14-31 restated for a scalar ODE
    un = u
    u1 = un + dt * L(u)
    u2 = 0.75 * un + 0.25 * u1 + 0.25 * dt * L(u1)
    return (1 / 3) * un + (2 / 3) * u2 + (2 / 3) * dt * L(u2)


def test_rk3_third_order():
    # test/test_rk3.jl:32-57
    def run(dt):
        y = 1.0
        for _ in range(round(1.0 / dt)):
            y = _rk3_generic(y, lambda u: -u, dt)
        return y
    e1 = abs(run(0.1) - math.exp(-1))
    e2 = abs(run(0.01) - math.exp(-1))
    assert e2 < 1e-6 and e1 / e2 > 100


def test_hllc_rotations_consistent(orc):
    # hllc_flux_y/z are argument permutations of the x solver (src/hllc.jl:176-208)
    L = (1.0, 0.3, -0.2, 0.1, 2.5)
    R = (0.4, -0.1, 0.25, 0.05, 0.9)
    fx = orc.hllc_flux(0, L, R, 1.4)
    Ly = (L[0], L[2], L[1], L[3], L[4])
    Ry = (R[0], R[2], R[1], R[3], R[4])
    fy = orc.hllc_flux(1, Ly, Ry, 1.4)
    assert fx[0] == fy[0] and fx[4] == fy[4]
    assert fx[1] == fy[2] and fx[2] == fy[1] and fx[3] == fy[3]


def test_hllc_uniform_state_is_physical_flux(orc):
    s = (1.0, 0.5, 0.0, 0.0, 2.5 + 0.125)
    f = orc.hllc_flux(0, s, s, 1.4)
    p = 0.4 * (s[4] - 0.5 * 0.25)
    assert f[0] == pytest.approx(0.5, rel=1e-15)
    assert f[1] == pytest.approx(0.25 + p, rel=1e-14)
    assert f[4] == pytest.approx((s[4] + p) * 0.5, rel=1e-14)


def test_blackhole_sink_radius_and_time(orc):
    # test/test_blackhole.jl:1-48
    bh = orc.make_bh((0, 0, 0), (0, 0.5, 0), 0.5, 1e-3, 485.0, 1e-3)
    assert orc.r_sink(bh) == 1e-3
    bh_nr = orc.make_bh((0, 0, 0), (0, 0, 0), 0.5, 1e-4, 1.0, 1e-4)
    rs = orc.r_sink(bh_nr)
    assert rs == pytest.approx(3.0)
    ts = orc.t_sink(bh_nr)
    assert ts == pytest.approx(rs / math.sqrt(2 * 0.5 / rs), rel=1e-12)


def test_ghost_fill_corner_composition(orc):
    # src/euler3d.jl:33-62: x then y then z fills make every ghost cell a copy
    # of the nearest (outflow) or wrapped (periodic) active cell.
    rng = np.random.default_rng(1)
    nx, ny, nz = 5, 4, 6
    for bc, fill in (("outflow", orc.fill_ghost_3d_outflow), ("periodic", orc.fill_ghost_3d_periodic)):
        U = np.asfortranarray(rng.standard_normal((5, nx + 6, ny + 6, nz + 6)))
        fill(U)
        def m(a, n):
            if bc == "outflow":
                return min(max(a, NG), NG + n - 1)
            return NG + ((a - NG) % n)
        for i in range(nx + 6):
            for j in range(ny + 6):
                for k in range(nz + 6):
                    src = (m(i, nx), m(j, ny), m(k, nz))
                    np.testing.assert_array_equal(U[:, i, j, k], U[(slice(None),) + src])
