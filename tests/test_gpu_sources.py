"""GPU parity of the source terms, the FFT Poisson solve and the coupled step
against the oracle (src/gravity_bh.jl, src/sinks.jl, src/self_gravity.jl,
scripts/run_sn50_fiducial.jl:756-818).

Pointwise sources and accretion are bit-identical.  FFT results and the
whole-grid gas-force sum are compared within 1e-12 (relative L-inf of the
field / of the sum of term magnitudes): the reference's own FFT (FFTW/cuFFT)
and its sequential sum differ from any other correct evaluation at that level.
"""
import math

import numpy as np
import pytest

from binary_ic import binary_setup
from gpu_util import NG, assert_bitwise, dev, host, random_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
TOL = 1e-12


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


def _bhs(lib, specs):
    return [lib.BlackHole(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"]) for s in specs]


def _obhs(orc, specs):
    return [orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"]) for s in specs]


SPECS = [dict(pos=(0.43, 0.37, 0.52), vel=(0.1, -0.2, 0.05), mass=1.0, eps=0.05, c_code=1e6, r_floor=0.3),
         dict(pos=(0.2, 0.61, 0.3), vel=(-0.1, 0.0, 0.2), mass=0.5, eps=0.02, c_code=1e6, r_floor=0.25)]


@pytest.mark.parametrize("torque_free", [True, False])
def test_bh_gravity_and_sinks_bitwise(orc, bsn, torque_free):
    n = (13, 9, 11)
    U = random_state(*n, seed=21)
    dU = np.asfortranarray(np.random.default_rng(22).standard_normal(U.shape))
    Ud, dUd = dev(U), dev(dU)
    args = (0.07, 0.08, 0.06)
    bsn.add_bh_gravity_source(dUd, Ud, *n, *args, _bhs(bsn, SPECS), 0.0, -0.1, 0.05)
    orc.add_bh_gravity_source(dU, U, *args, _obhs(orc, SPECS), 0.0, -0.1, 0.05)
    assert_bitwise(host(dUd), dU, "bh gravity")
    bsn.add_sink_sources(dUd, Ud, *n, *args, _bhs(bsn, SPECS), 0.0, -0.1, 0.05, f_sink=1.3, torque_free=torque_free,
                         rho_sink_min=0.9)
    orc.add_sink_sources(dU, U, *args, _obhs(orc, SPECS), 0.0, -0.1, 0.05, f_sink=1.3, torque_free=torque_free,
                         rho_sink_min=0.9)
    assert_bitwise(host(dUd), dU, "sinks")


def test_accrete_bitwise_and_gas_force(orc, bsn):
    n = (16, 14, 12)
    U = random_state(*n, seed=23)
    Ud = dev(U)
    args = (0.05, 0.05, 0.05)
    for s in SPECS:
        bg = bsn.BlackHole(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"])
        bo = orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"])
        bsn.accrete(bg, Ud, *n, *args, 0.0, 0.0, 0.0, 1e-3, f_sink=1.1, rho_sink_min=0.5)
        orc.accrete(bo, U, *args, 0.0, 0.0, 0.0, 1e-3, f_sink=1.1, rho_sink_min=0.5)
        assert bg.mass == bo.mass and list(bg.vel) == list(bo.vel)
        Fg = bsn.gas_force_on_bh(Ud, *n, *args, bg, 0.0, 0.0, 0.0)
        Fo = orc.gas_force_on_bh(U, *args, bo, 0.0, 0.0, 0.0)
        # scale: sum of |terms| of the reference's sequential sum
        c = [(np.arange(m) + 0.5) * 0.05 for m in n]
        X, Y, Z = np.meshgrid(*c, indexing="ij")
        d = np.stack([X - s["pos"][0], Y - s["pos"][1], Z - s["pos"][2]])
        r2 = (d ** 2).sum(0) + s["eps"] ** 2
        rho = U[0, NG:NG + n[0], NG:NG + n[1], NG:NG + n[2]]
        mag = (np.abs(s["mass"] / (r2 * np.sqrt(r2)) * rho * 0.05 ** 3 * d)).sum(axis=(1, 2, 3))
        assert np.all(np.abs(Fg - Fo) <= TOL * mag)


def _sphere(n, dx, R):
    c = (np.arange(n) + 0.5) * dx - 0.5
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    return np.asfortranarray(np.where(np.sqrt(X ** 2 + Y ** 2 + Z ** 2) < R, 1.0, 0.0))


@pytest.mark.parametrize("shape", [(32, 32, 32), (16, 32, 8), (64, 64, 64)])
def test_poisson_matches_oracle(orc, bsn, shape):
    rng = np.random.default_rng(24)
    rho = np.asfortranarray(rng.random(shape))
    d = (0.03, 0.02, 0.05)
    phi_o = orc.solve_poisson_isolated(rho, *d)
    phi_g = host(bsn.solve_poisson_isolated(dev(rho), *shape, *d))
    assert np.abs(phi_g - phi_o).max() <= TOL * np.abs(phi_o).max()


def test_poisson_known_answers_on_gpu(bsn):
    # test/test_self_gravity.jl:29-131 and docs/phase7.md (0.49 %, 3.5 %, 8.1 %)
    def ratio_err(N):
        dx = 1.0 / N
        phi = host(bsn.solve_poisson_isolated(dev(_sphere(N, dx, 0.15)), N, N, N, dx, dx, dx))
        jc = round(0.5 / dx + 0.5)
        r = lambda i: math.sqrt(((i - 0.5) * dx - 0.5) ** 2 + 2 * ((jc - 0.5) * dx - 0.5) ** 2)
        iA, iB = round(0.75 / dx + 0.5), round(0.85 / dx + 0.5)
        num = phi[iA - 1, jc - 1, jc - 1] / phi[iB - 1, jc - 1, jc - 1]
        return abs(num - r(iB) / r(iA)) / (r(iB) / r(iA))
    e16, e32 = ratio_err(16), ratio_err(32)
    assert e32 < e16 and round(e32, 4) == 0.0049 and round(e16, 3) == 0.035
    N, dx = 32, 1 / 32
    rho = _sphere(N, dx, 0.15)
    M = rho.sum() * dx ** 3
    phi = host(bsn.solve_poisson_isolated(dev(rho), N, N, N, dx, dx, dx))
    Ea = -3 * M ** 2 / (5 * 0.15)
    assert round(abs((0.5 * (rho * phi).sum() * dx ** 3 - Ea) / Ea), 3) == 0.081


def test_sg_gradient_bitwise_and_source(orc, bsn):
    n = (16, 16, 16)
    U = random_state(*n, seed=25)
    dU = np.zeros_like(U, order="F")
    phi = orc.solve_poisson_isolated(np.asfortranarray(U[0, NG:-NG, NG:-NG, NG:-NG]), 0.1, 0.1, 0.1)
    Ud, dUd = dev(U), dev(dU)
    bsn.apply_sg_force_level(dUd, Ud, dev(phi), *n, 0.1, 0.1, 0.1)
    orc.sg_gradient(dU, U, phi, 0.1, 0.1, 0.1)
    assert_bitwise(host(dUd), dU, "sg gradient")
    dU2 = np.zeros_like(U, order="F")
    dUd2 = dev(dU2)
    bsn.add_self_gravity_source(dUd2, Ud, *n, 0.1, 0.1, 0.1)
    orc.add_self_gravity_source(dU2, U, 0.1, 0.1, 0.1)
    g = host(dUd2)
    assert np.abs(g - dU2).max() <= TOL * np.abs(dU2).max()


@pytest.mark.parametrize("sinks_on", [True, False])
@pytest.mark.parametrize("torque_free", [True, False])
def test_coupled_step_kinematic_orbit_bitwise(orc, bsn, sinks_on, torque_free):
    # orbit driven kinematically (kepler_update!, run_sn30_fixedorbit.jl), so
    # the whole step is pointwise arithmetic plus the exact-order accretion
    U, dx, x0, specs = binary_setup(orc, n=32)
    Ud = dev(U)
    bg, bo = _bhs(bsn, specs), orc.bh_array(_obhs(orc, specs))
    orbit_g = bsn.KeplerOrbit(bg)
    orbit_o = orc.kepler_init(bo)
    t = 0.0
    for _ in range(3):
        dt = orc.cfl_dt_3d(U, dx, dx, dx, 4 / 3, 0.4)
        assert bsn.cfl_dt_3d(Ud, 32, 32, 32, dx, dx, dx, 4 / 3, 0.4) == dt
        bsn.kepler_update(bg, orbit_g, t + dt)
        orc.kepler_update(bo, orbit_o, t + dt)
        ton = -1.0 if sinks_on else 1e9
        bsn.coupled_step(Ud, bg, dt, t, 32, 32, 32, dx, x0, x0, x0, 4 / 3, 1.0, 1e-8, 1e-10, torque_free, False, ton,
                         2e-8, evolve_orbit=False)
        orc.coupled_step(U, bo, 2, dt, t, dx, x0, x0, x0, 4 / 3, 1.0, 1e-8, 1e-10, torque_free, False, ton, 2e-8,
                         evolve_orbit=False)
        t += dt
        assert_bitwise(host(Ud), U, "coupled step U")
        for i in range(2):
            assert bg[i].mass == bo[i].mass and list(bg[i].vel) == list(bo[i].vel)
            assert list(bg[i].pos) == list(bo[i].pos)


@pytest.mark.parametrize("self_gravity", [False, True])
def test_coupled_step_live_orbit(orc, bsn, self_gravity):
    # live N-body orbit (gas force from the whole-grid sum) and optional
    # self-gravity: within 1e-12 relative L-inf after each step
    U, dx, x0, specs = binary_setup(orc, n=32)
    Ud = dev(U)
    bg, bo = _bhs(bsn, specs), orc.bh_array(_obhs(orc, specs))
    t = 0.0
    for _ in range(2):
        dt = orc.cfl_dt_3d(U, dx, dx, dx, 4 / 3, 0.4)
        Fg = bsn.coupled_step(Ud, bg, dt, t, 32, 32, 32, dx, x0, x0, x0, 4 / 3, 1.0, 1e-8, 1e-10, True, self_gravity,
                              0.0, 2e-8, evolve_orbit=True)
        Fo = orc.coupled_step(U, bo, 2, dt, t, dx, x0, x0, x0, 4 / 3, 1.0, 1e-8, 1e-10, True, self_gravity, 0.0, 2e-8,
                              evolve_orbit=True)
        t += dt
        G = host(Ud)
        for q in range(5):
            assert np.abs(G[q] - U[q]).max() <= TOL * np.abs(U[q]).max(), q
        assert np.allclose(Fg, Fo, rtol=1e-10, atol=1e-14 * np.abs(Fo).max())
        for i in range(2):
            assert abs(bg[i].mass - bo[i].mass) <= 1e-13 * bo[i].mass
            assert np.allclose(list(bg[i].pos), list(bo[i].pos), rtol=0, atol=1e-13)


def _reference_coupled_loop(orc, U, bo, dx, x0, steps, evolve, self_gravity, ton=0.0):
    t = 0.0
    for _ in range(steps):
        dt = orc.cfl_dt_3d(U, dx, dx, dx, 4 / 3, 0.4)
        orc.coupled_step(U, bo, 2, dt, t, dx, x0, x0, x0, 4 / 3, 1.0, 1e-8, 1e-10, True, self_gravity, ton, 2e-8,
                         evolve_orbit=evolve)
        t += dt
    return t


@pytest.mark.parametrize("ton", [0.0, 1e9])
def test_coupled_run_steps_static_bhs_bitwise(orc, bsn, ton):
    """The device-resident coupled loop (dt on the device, one graph per step)
    against the reference driver loop: bit-identical state, BH masses and
    velocities with the orbit frozen (accretion still changes them)."""
    U, dx, x0, specs = binary_setup(orc, n=32)
    Ud = dev(U)
    bg, bo = _bhs(bsn, specs), orc.bh_array(_obhs(orc, specs))
    t_ref = _reference_coupled_loop(orc, U, bo, dx, x0, 3, False, False, ton)
    t, n = bsn.coupled_run_steps(Ud, bg, 32, 32, 32, dx, x0, x0, x0, 4 / 3, 0.4, n_steps=3, f_sink=1.0,
                                 rho_floor=1e-8, P_floor=1e-10, torque_free=True, t_bh2_sink_on=ton,
                                 rho_sink_min=2e-8, evolve_orbit=False)
    assert n == 3 and t == t_ref
    assert_bitwise(host(Ud), U, "coupled loop U")
    for i in range(2):
        assert bg[i].mass == bo[i].mass and list(bg[i].vel) == list(bo[i].vel) and list(bg[i].pos) == list(bo[i].pos)


@pytest.mark.parametrize("self_gravity", [False, True])
def test_coupled_run_steps_live_orbit(orc, bsn, self_gravity):
    """Live N-body orbit on the device: within the whole-grid gas-force
    summation's rounding of the reference driver loop (as the single step)."""
    U, dx, x0, specs = binary_setup(orc, n=32)
    Ud = dev(U)
    bg, bo = _bhs(bsn, specs), orc.bh_array(_obhs(orc, specs))
    t_ref = _reference_coupled_loop(orc, U, bo, dx, x0, 2, True, self_gravity)
    t, n = bsn.coupled_run_steps(Ud, bg, 32, 32, 32, dx, x0, x0, x0, 4 / 3, 0.4, n_steps=2, f_sink=1.0,
                                 rho_floor=1e-8, P_floor=1e-10, torque_free=True, self_gravity=self_gravity,
                                 rho_sink_min=2e-8, evolve_orbit=True)
    assert n == 2 and abs(t - t_ref) <= 1e-12 * t_ref
    G = host(Ud)
    for q in range(5):
        assert np.abs(G[q] - U[q]).max() <= TOL * np.abs(U[q]).max(), q
    for i in range(2):
        assert abs(bg[i].mass - bo[i].mass) <= 1e-13 * bo[i].mass
        assert np.allclose(list(bg[i].pos), list(bo[i].pos), rtol=0, atol=1e-13)


def test_coupled_run_steps_t_end_and_fp32(orc, bsn):
    """t_end stops the loop exactly; FP32 stencils stay close to FP64."""
    U, dx, x0, specs = binary_setup(orc, n=32)
    U64, U32 = dev(U), dev(U)
    b64, b32 = _bhs(bsn, specs), _bhs(bsn, specs)
    t_end = 2.5 * orc.cfl_dt_3d(U, dx, dx, dx, 4 / 3, 0.4)
    kw = dict(n_steps=1000, t_end=t_end, f_sink=1.0, rho_floor=1e-8, P_floor=1e-10, rho_sink_min=2e-8)
    t64, n64 = bsn.coupled_run_steps(U64, b64, 32, 32, 32, dx, x0, x0, x0, 4 / 3, 0.4, **kw)
    t32, n32 = bsn.coupled_run_steps(U32, b32, 32, 32, 32, dx, x0, x0, x0, 4 / 3, 0.4, precision="f32", **kw)
    assert t64 == t_end and t32 == t_end and n64 >= 3
    a = (0,) + (slice(NG, -NG),) * 3
    A, B = host(U32)[a], host(U64)[a]
    assert np.abs(A - B).sum() / np.abs(B).sum() < 1e-5


def test_diagnostics_device_reduction(orc, bsn):
    """bsn_diagnostics_f64 (one compensated device reduction) against the
    oracle's restatement of src/diagnostics.jl, within 1e-13 of the sum of
    magnitudes."""
    U, dx, x0, specs = binary_setup(orc, n=32)
    t = 0.0
    bo = orc.bh_array(_obhs(orc, specs))
    dt = orc.cfl_dt_3d(U, dx, dx, dx, 4 / 3, 0.4)
    orc.coupled_step(U, bo, 2, dt, t, dx, x0, x0, x0, 4 / 3, 1.0, 1e-8, 1e-10, True, False, 0.0, 2e-8,
                     evolve_orbit=True)   # a state with motion
    obhs = [bo[i] for i in range(2)]
    gbhs = [bsn.BlackHole(list(b.pos), list(b.vel), b.mass, b.eps, b.c_code, b.r_floor) for b in obhs]
    ref = orc.diagnostics(U, dx, dx, dx, x0, x0, x0, obhs, 4 / 3)
    got = bsn.diagnostics(dev(U), 32, 32, 32, dx, dx, dx, x0, x0, x0, gbhs, 4 / 3)
    a = (slice(NG, -NG),) * 3
    mag = np.abs(U[(4,) + a]).sum() + np.abs(U[(0,) + a]).sum() + np.abs(U[(1,) + a]).sum() + \
        np.abs(U[(2,) + a]).sum() + np.abs(U[(3,) + a]).sum()
    assert np.all(np.abs(got - ref) <= 1e-13 * mag * dx ** 3), (got, ref)
    assert ref[8] > 0


def test_coupled_run_steps_records_diagnostics(orc, bsn):
    """The device loop's per-step records: {t, dt, diagnostics} equal to the
    standalone reduction of the end state (same kernel), times and dts of the
    reference loop."""
    U, dx, x0, specs = binary_setup(orc, n=32)
    Ud = dev(U)
    bg = _bhs(bsn, specs)
    rec = torch.zeros((4, bsn.DIAG_RECORD), dtype=torch.float64, device="cuda")
    t, n = bsn.coupled_run_steps(Ud, bg, 32, 32, 32, dx, x0, x0, x0, 4 / 3, 0.4, n_steps=3, f_sink=1.0,
                                 rho_floor=1e-8, P_floor=1e-10, rho_sink_min=2e-8, evolve_orbit=False, diag=rec)
    R = rec.cpu().numpy()
    assert n == 3 and R[2, 0] == t and np.all(R[3] == 0.0)
    assert np.all(R[:3, 1] > 0) and R[0, 0] == R[0, 1] and R[1, 0] == R[0, 0] + R[1, 1]
    end = bsn.diagnostics(Ud, 32, 32, 32, dx, dx, dx, x0, x0, x0, bg, 4 / 3)
    assert np.array_equal(R[2, 2:12], end)
    # the reference loop's times
    bo = orc.bh_array(_obhs(orc, specs))
    t_ref = 0.0
    for k in range(3):
        dt = orc.cfl_dt_3d(U, dx, dx, dx, 4 / 3, 0.4)
        assert dt == R[k, 1]
        orc.coupled_step(U, bo, 2, dt, t_ref, dx, x0, x0, x0, 4 / 3, 1.0, 1e-8, 1e-10, True, False, 0.0, 2e-8,
                         evolve_orbit=False)
        t_ref += dt
    assert t_ref == t
