"""GPU parity of the FP64 uniform-grid path against the oracle: ghost fills,
floors, euler3d_rhs!, euler3d_step!, cfl_dt_3d -- bit for bit on the whole
ghosted array (the reference's CPU arithmetic is reproduced exactly)."""
import numpy as np
import pytest

from gpu_util import NG, assert_bitwise, dev, host, random_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SIZES = [(13, 7, 5), (16, 16, 16), (24, 9, 17)]


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_ghost_fill(orc, bsn, n, bc):
    U = random_state(*n, seed=1)
    Ud = dev(U)
    (bsn.fill_ghost_3d_outflow if bc == "outflow" else bsn.fill_ghost_3d_periodic)(Ud, *n)
    (orc.fill_ghost_3d_outflow if bc == "outflow" else orc.fill_ghost_3d_periodic)(U)
    assert_bitwise(host(Ud), U, "ghost fill")


def test_floors(orc, bsn):
    n = (13, 7, 5)
    U = random_state(*n, seed=2, vacuum=True)
    Ud = dev(U)
    bsn.apply_floors_3d(Ud, *n, 1e-6, 1e-4, 1.4)
    orc.apply_floors_3d(U, 1e-6, 1e-4, 1.4)
    assert_bitwise(host(Ud), U, "floors")


@pytest.mark.parametrize("n", SIZES + [(32, 4, 4)])
@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_euler3d_rhs(orc, bsn, n, bc):
    U = random_state(*n, seed=3, vacuum=True)
    dx, dy, dz = 0.1, 0.07, 0.13
    Fx, Fy, Fz = orc.flux_arrays(*n)
    dU = np.zeros_like(U, order="F")
    Ud = dev(U)
    dUd = torch.full_like(Ud, 7.0)
    Fxd, Fyd, Fzd = (torch.full_like(dev(a), 3.0) for a in (Fx, Fy, Fz))
    bsn.euler3d_rhs(dUd, Fxd, Fyd, Fzd, Ud, *n, dx, dy, dz, 1.4, bc=bc, rho_floor=1e-6, P_floor=1e-4)
    orc.euler3d_rhs(dU, Fx, Fy, Fz, U, dx, dy, dz, 1.4, bc=bc, rho_floor=1e-6, P_floor=1e-4)
    assert_bitwise(host(Ud), U, "U after rhs (ghosts+floors)")
    assert_bitwise(host(dUd), dU, "dU")
    assert_bitwise(host(Fxd), Fx, "Fx")
    assert_bitwise(host(Fyd), Fy, "Fy")
    assert_bitwise(host(Fzd), Fz, "Fz")


def test_euler3d_rhs_with_many_floored_cells_is_deterministic(orc, bsn):
    """euler3d_rhs! floors U in place; with thousands of blocks staging one
    another's cells, U is floored only after the flux launch, so no block
    stages a half-floored cell: every call equals the oracle (FP64) and the
    FP32 right-hand side repeats bit for bit."""
    n = (96, 80, 72)
    U = random_state(*n, seed=31, vacuum=True)
    rng = np.random.default_rng(32)
    a = (slice(NG, -NG),) * 3
    neg = rng.random(U[0][a].shape) < 0.15
    U[0][a][neg] *= -1.0   # negative densities: the floors' first branch
    orc.fill_ghost_3d_outflow(U)
    d = (0.01, 0.011, 0.012)
    kw = dict(rho_floor=1e-6, P_floor=1e-4)
    Fo = orc.flux_arrays(*n)
    dUo, Uo = np.zeros_like(U, order="F"), U.copy(order="F")
    orc.euler3d_rhs(dUo, *Fo, Uo, *d, 1.4, fill_ghosts=False, **kw)
    f32 = []
    for _ in range(3):
        Ud, dUd = dev(U), torch.zeros_like(dev(U))
        Fd = [torch.zeros_like(dev(f)) for f in Fo]
        bsn.euler3d_rhs(dUd, *Fd, Ud, *n, *d, 1.4, fill_ghosts=False, **kw)
        assert_bitwise(host(Ud), Uo, "U after rhs")
        assert_bitwise(host(dUd), dUo, "dU")
        for f, g in zip(Fd, Fo):
            assert_bitwise(host(f), g, "F")
        U32, dU32 = dev(U), torch.zeros_like(dev(U))
        bsn.euler3d_rhs_f32(dU32, None, None, None, U32, *n, *d, 1.4, fill_ghosts=False, **kw)
        assert torch.equal(U32, Ud)
        f32.append(dU32)
    assert torch.equal(f32[0], f32[1]) and torch.equal(f32[0], f32[2])


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_euler3d_step_random(orc, bsn, n, bc):
    U = random_state(*n, seed=4, vacuum=True)
    Ud = dev(U)
    args = (0.1, 0.07, 0.13, 2e-3, 1.4)
    bsn.euler3d_step(Ud, *n, *args, bc=bc, rho_floor=1e-6, P_floor=1e-4)
    orc.euler3d_step(U, *args, bc=bc, rho_floor=1e-6, P_floor=1e-4)
    assert_bitwise(host(Ud), U, "U after step")


def test_step_sod64_and_cfl(orc, bsn):
    # 3D Sod 64^3 (gamma 1.4, CFL 0.4): one full RK3 step from the initial state
    U, dims, (dx, dy, dz) = orc.sod_ic_3d("x", n_normal=64, n_trans=64)
    Ud = dev(U)
    dt_g = bsn.cfl_dt_3d(Ud, *dims, dx, dy, dz, 1.4, 0.4)
    dt_o = orc.cfl_dt_3d(U, dx, dy, dz, 1.4, 0.4)
    assert dt_g == dt_o
    bsn.euler3d_step(Ud, *dims, dx, dy, dz, dt_g, 1.4)
    orc.euler3d_step(U, dx, dy, dz, dt_o, 1.4)
    assert_bitwise(host(Ud), U, "Sod 64^3 step")
    assert bsn.cfl_dt_3d(Ud, *dims, dx, dy, dz, 1.4, 0.4) == orc.cfl_dt_3d(U, dx, dy, dz, 1.4, 0.4)


def test_sedov_run_bitwise(orc, bsn):
    # Sedov 32^3 on [-1,1]^3 to t=0.1 (test/test_sedov.jl): every step bitwise
    g, n, L = 5 / 3, 32, 1.0
    dx = 2 * L / n
    U = orc.state(n, n, n)
    orc.sedov_ic_3d(U, dx, dx, dx, g, E_blast=1.0, rho_bg=1.0, P_floor=1e-5, x_offset=-L, y_offset=-L, z_offset=-L)
    Ud = dev(U)
    t = 0.0
    while t < 0.1:
        dt = min(orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4), 0.1 - t)
        assert bsn.cfl_dt_3d(Ud, n, n, n, dx, dx, dx, g, 0.4) == orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4)
        orc.euler3d_step(U, dx, dx, dx, dt, g, rho_floor=1e-6, P_floor=1e-6)
        bsn.euler3d_step(Ud, n, n, n, dx, dx, dx, dt, g, rho_floor=1e-6, P_floor=1e-6)
        t += dt
    assert_bitwise(host(Ud), U, "Sedov 32^3 end state")


def test_sod_L1_on_gpu_matches_documented(orc, bsn):
    from analytic import sod_errors
    for d in "xyz":
        U, dims, (dx, dy, dz) = orc.sod_ic_3d(d)
        Ud = dev(U)
        t = 0.0
        while t < 0.2:
            dt = min(bsn.cfl_dt_3d(Ud, *dims, dx, dy, dz, 1.4, 0.4), 0.2 - t)
            bsn.euler3d_step(Ud, *dims, dx, dy, dz, dt, 1.4)
            t += dt
        e = sod_errors(host(Ud), d, dims, (dx, dy, dz)["xyz".index(d)], 0.2)
        assert (round(e[0], 4), round(e[1], 4), round(e[2], 4)) == (0.0038, 0.0073, 0.0031)


def test_bad_arguments_raise(bsn):
    U = bsn.state(8, 8, 8)
    with pytest.raises(ValueError):
        bsn.euler3d_step(U, 8, 8, 9, 0.1, 0.1, 0.1, 1e-3, 1.4)
    with pytest.raises(bsn.BSNError):
        bsn.euler3d_step(bsn.state(2, 2, 2), 2, 2, 2, 0.1, 0.1, 0.1, 1e-3, 1.4, bc="periodic")
