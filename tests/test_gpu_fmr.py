"""GPU parity of the two-level FMR path against the oracle (src/fmr3d.jl,
src/fmr_gravity.jl): prolongation, restriction, fmr3d_step! (coarse RK3 with
flux registers, fine subcycles, restriction, Berger-Colella correction) and
cfl_dt_fmr3d are bit-identical; steps with self-gravity match within 1e-12
(the FFT)."""
import numpy as np
import pytest

from gpu_util import NG, assert_bitwise, dev, host, random_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


def _pair(orc, bsn, Uc, dxc, lo, hi, ratio, gamma, **kw):
    """Build the oracle grid and the device grid from the same coarse state."""
    n = orc.dims(Uc)
    Go = orc.FMRGrid(Uc.copy(order="F"), dxc, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], ratio, gamma, **kw)
    Gd = bsn.FMRGrid3D(dev(Uc), *n, dxc, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], ratio, gamma, **kw)
    return Go, Gd


def _sedov_fmr(orc, bsn):
    # test/test_fmr3d.jl:113-170: 8^3 coarse on [-0.5,0.5]^3, fine 16^3, ratio 4
    g, nc, L, ratio = 5 / 3, 8, 0.5, 4
    dxc = 2 * L / nc
    dxf = dxc / ratio
    Uc = orc.state(nc, nc, nc)
    orc.sedov_ic_3d(Uc, dxc, dxc, dxc, g, E_blast=1.0, r_inject=0.15, rho_bg=1.0, P_floor=1e-5,
                    x_offset=-L, y_offset=-L, z_offset=-L)
    orc.fill_ghost_3d_outflow(Uc)
    Go, Gd = _pair(orc, bsn, Uc, dxc, (3, 3, 3), (6, 6, 6), ratio, g, rho_floor=1e-10, P_floor=1e-5)
    xflo = 2 * dxc - L
    orc.sedov_ic_3d(Go.Uf, dxf, dxf, dxf, g, E_blast=1.0, r_inject=0.15, rho_bg=1.0, P_floor=1e-5,
                    x_offset=xflo, y_offset=xflo, z_offset=xflo)
    Go.prolong_fine_ghosts()
    Gd.Uf.copy_(dev(Go.Uf))
    return Go, Gd


def test_prolong_all_and_ghosts_and_restrict(orc, bsn):
    Uc = random_state(16, 12, 14, seed=31)
    Go, Gd = _pair(orc, bsn, Uc, 0.1, (6, 5, 6), (10, 7, 8), 2, 1.4)
    assert_bitwise(host(Gd.Uf), Go.Uf, "prolong_all")
    Uf = random_state(*orc.dims(Go.Uf), seed=32)
    Go.Uf[...] = Uf
    Gd.Uf.copy_(dev(Uf))
    Go.prolong_fine_ghosts()
    Gd.prolong_fine_ghosts()
    assert_bitwise(host(Gd.Uf), Go.Uf, "prolong_fine_ghosts")
    Go.restrict()
    Gd.restrict()
    assert_bitwise(host(Gd.Uc), Go.Uc, "restrict")


def test_fmr_sedov_run_bitwise_and_documented_L1(orc, bsn):
    Go, Gd = _sedov_fmr(orc, bsn)
    t, steps = 0.0, 0
    while t < 0.01:
        dt = Go.cfl_dt(0.4)
        assert bsn.cfl_dt_fmr3d(Gd, 0.4) == dt
        dt = min(dt, 0.01 - t)
        Go.step(dt)
        bsn.fmr3d_step(Gd, dt)
        t += dt
        steps += 1
        assert_bitwise(host(Gd.Uc), Go.Uc, f"coarse after step {steps}")
        assert_bitwise(host(Gd.Uf), Go.Uf, f"fine after step {steps}")
    assert steps >= 2


@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_fmr_ratio2_random_bitwise(orc, bsn, bc):
    Uc = random_state(16, 16, 12, seed=33, gamma=5 / 3)
    if bc == "outflow":
        orc.fill_ghost_3d_outflow(Uc)
    else:
        orc.fill_ghost_3d_periodic(Uc)
    Go, Gd = _pair(orc, bsn, Uc, 0.0625, (6, 6, 5), (11, 10, 8), 2, 5 / 3, bc=bc, rho_floor=1e-8, P_floor=1e-6)
    for _ in range(2):
        dt = Go.cfl_dt(0.3)
        assert bsn.cfl_dt_fmr3d(Gd, 0.3) == dt
        Go.step(dt)
        bsn.fmr3d_step(Gd, dt)
    assert_bitwise(host(Gd.Uc), Go.Uc, "coarse")
    assert_bitwise(host(Gd.Uf), Go.Uf, "fine")


def _sg_grid(orc, bsn, nc=8, L=0.5, ratio=4, R=0.2, rbg=1e-4, e=1e-3, g=5 / 3):
    dxc = 2 * L / nc
    Uc = orc.state(nc, nc, nc)
    c = (np.arange(nc) + 0.5) * dxc - L
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    rho = np.where(np.sqrt(X ** 2 + Y ** 2 + Z ** 2) < R, 1.0, rbg)
    a = (slice(NG, NG + nc),) * 3
    Uc[(0,) + a] = rho
    Uc[(4,) + a] = rho * e
    orc.fill_ghost_3d_outflow(Uc)
    lo, hi = nc // 4 + 1, 3 * (nc // 4)
    Go, Gd = _pair(orc, bsn, Uc, dxc, (lo,) * 3, (hi,) * 3, ratio, g, rho_floor=1e-12, P_floor=1e-12)
    dxf = dxc / ratio
    nf = (hi - lo + 1) * ratio
    cf = (np.arange(nf) + 0.5) * dxf + (lo - 1) * dxc - L
    X, Y, Z = np.meshgrid(cf, cf, cf, indexing="ij")
    rf = np.where(np.sqrt(X ** 2 + Y ** 2 + Z ** 2) < R, 1.0, rbg)
    af = (slice(NG, NG + nf),) * 3
    Go.Uf[(0,) + af] = rf
    Go.Uf[(4,) + af] = rf * e
    Go.prolong_fine_ghosts()
    Gd.Uf.copy_(dev(Go.Uf))
    return Go, Gd


def test_fmr_poisson_matches_oracle(orc, bsn):
    # solve_fmr_poisson on the reference's sphere grid (test/test_fmr_gravity.jl:242-260)
    Go, Gd = _sg_grid(orc, bsn)
    pc_o, pf_o = Go.solve_poisson()
    pc_d, pf_d = bsn.solve_fmr_poisson(Gd)
    assert_bitwise(host(Gd.Uc), Go.Uc, "restricted density")
    assert np.abs(host(pc_d) - pc_o).max() <= 1e-12 * np.abs(pc_o).max()
    assert np.abs(host(pf_d) - pf_o).max() <= 1e-12 * np.abs(pf_o).max()


def _smooth_sg_grid(orc, bsn, nc=16, L=0.5, ratio=2, lo=6, hi=11, sigma=0.15, g=5 / 3):
    # a well-conditioned self-gravitating blob: Gaussian density, no
    # prolongation overshoot to rho <= 0 (where the reference's HLLC switches
    # branch discontinuously and FFT-rounding-level differences in Phi would
    # be amplified)
    dxc = 2 * L / nc
    Uc = orc.state(nc, nc, nc)
    c = (np.arange(nc) + 0.5) * dxc - L
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    rho = 1e-2 + np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / (2 * sigma ** 2))
    a = (slice(NG, NG + nc),) * 3
    Uc[(0,) + a] = rho
    Uc[(4,) + a] = rho * 1e-2
    orc.fill_ghost_3d_outflow(Uc)
    Go, Gd = _pair(orc, bsn, Uc, dxc, (lo,) * 3, (hi,) * 3, ratio, g, rho_floor=1e-12, P_floor=1e-12)
    dxf = dxc / ratio
    nf = (hi - lo + 1) * ratio
    cf = (np.arange(nf) + 0.5) * dxf + (lo - 1) * dxc - L
    X, Y, Z = np.meshgrid(cf, cf, cf, indexing="ij")
    rf = 1e-2 + np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / (2 * sigma ** 2))
    af = (slice(NG, NG + nf),) * 3
    Go.Uf[(0,) + af] = rf
    Go.Uf[(4,) + af] = rf * 1e-2
    Go.prolong_fine_ghosts()
    Gd.Uf.copy_(dev(Go.Uf))
    return Go, Gd


@pytest.mark.parametrize("G_grav", [1.0, 0.5])
def test_fmr_selfgravity_steps_match_oracle(orc, bsn, G_grav):
    Go, Gd = _smooth_sg_grid(orc, bsn)
    for _ in range(2):
        dt = Go.cfl_dt(0.4)
        Go.step(dt, self_gravity=True, G_grav=G_grav)
        bsn.fmr3d_step(Gd, dt, self_gravity=True, G_grav=G_grav)
        for A, B in ((host(Gd.Uc), Go.Uc), (host(Gd.Uf), Go.Uf)):
            for q in range(5):
                scale = max(np.abs(B[q]).max(), 1e-300)
                assert np.abs(A[q] - B[q]).max() <= 1e-12 * scale, q


def test_fmr_selfgravity_reference_assertions_on_gpu(orc, bsn):
    # test/test_fmr_gravity.jl:229-323 run through the device path
    Go, Gd = _sg_grid(orc, bsn)
    G2 = _sg_grid(orc, bsn)[1]
    bsn.fmr3d_step(Gd, 1e-4)
    bsn.fmr3d_step(G2, 1e-4, self_gravity=False)
    assert torch.equal(Gd.Uc, G2.Uc) and torch.equal(Gd.Uf, G2.Uf)
    _, Gd = _sg_grid(orc, bsn)
    bsn.fmr3d_step(Gd, 1e-4, self_gravity=True)
    Uc, Uf = host(Gd.Uc), host(Gd.Uf)
    nc, nf = Gd.coarse_dims[0], Gd.fine_dims[0]
    ac, af = (slice(NG, NG + nc),) * 3, (slice(NG, NG + nf),) * 3
    Mc = Uc[(0,) + ac].sum()
    for q in (1, 2, 3):
        assert abs(Uc[(q,) + ac].sum()) / Mc < 1e-10
        assert abs(Uf[(q,) + af].sum()) / Mc < 1e-10
    _, Gd = _sg_grid(orc, bsn, rbg=1e-6, e=1e-4)
    bsn.fmr3d_step(Gd, 5e-4, self_gravity=True)
    Uf = host(Gd.Uf)
    dxc = 1.0 / nc
    dxf = dxc / 4
    cf = (np.arange(nf) + 0.5) * dxf + (nc // 4) * dxc - 0.5
    X, Y, Z = np.meshgrid(cf, cf, cf, indexing="ij")
    r = np.maximum(np.sqrt(X ** 2 + Y ** 2 + Z ** 2), 1e-300)
    rad = (Uf[(1,) + af] * X + Uf[(2,) + af] * Y + Uf[(3,) + af] * Z) / r
    assert rad.sum() * dxf ** 3 < 0.0


def test_fmr_patch_too_close_to_boundary_is_rejected(bsn):
    # ratio 2 with the patch starting at coarse cell 1: the fine ghosts'
    # Lagrange stencil would read before the coarse array (checked on the host)
    U = bsn.state(8, 8, 8)
    with pytest.raises(bsn.BSNError):
        bsn.FMRGrid3D(U, 8, 8, 8, 0.1, 1, 4, 1, 4, 1, 4, 2, 1.4)
