"""The coupled driver loop on nested FMR levels on the device
(bsn_coupled_nested_run_steps) against the oracle's restatement
(orc_coupled_fmrN_step: composite gas force, nbody_step!, one nested step with
BH gravity / self-gravity / sinks on every level, accrete! from the finest
level), on three nested 16^3 levels of the binary-BH workload.  With the orbit
frozen every level, BH mass and BH velocity are bit-identical; a live orbit
and self-gravity agree within the rounding of the whole-grid gas-force and
FFT sums."""
import numpy as np
import pytest

from binary_ic import binary_nested_setup
from gpu_util import NG, assert_bitwise, dev, host

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


def _setup(orc, bsn):
    H, boxes, dx0, x0, specs = binary_nested_setup(orc)
    n = H.levels[0].shape[1] - 2 * NG
    Hd = bsn.FMRHierarchy3D(dev(H.levels[0]), n, n, n, dx0, boxes, 4 / 3, rho_floor=1e-8, P_floor=1e-10,
                            init=False)
    for Ud, Uo in zip(Hd.levels, H.levels):
        Ud.copy_(dev(Uo))
    bo = orc.bh_array([orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"])
                       for s in specs])
    bg = [bsn.BlackHole(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"]) for s in specs]
    return H, Hd, bo, bg, x0


def _oracle_loop(H, bo, x0, steps, evolve, sg, ton=0.0, dt_max=0.0):
    t = 0.0
    for _ in range(steps):
        dt = H.cfl_dt(0.4)
        if dt_max > 0:
            dt = min(dt, dt_max)
        H.coupled_step(bo, 2, dt, t, x0, x0, x0, 1.0, True, sg, ton, 2e-8, evolve_orbit=evolve)
        t += dt
    return t


@pytest.mark.parametrize("ton", [0.0, 1e9])
def test_nested_coupled_static_bhs_bitwise(orc, bsn, ton):
    H, Hd, bo, bg, x0 = _setup(orc, bsn)
    t_ref = _oracle_loop(H, bo, x0, 3, False, False, ton)
    t, n = bsn.coupled_nested_run_steps(Hd, bg, x0, x0, x0, 0.4, n_steps=3, f_sink=1.0, torque_free=True,
                                        t_bh2_sink_on=ton, rho_sink_min=2e-8, evolve_orbit=False)
    assert n == 3 and t == t_ref
    for k, (Ud, Uo) in enumerate(zip(Hd.levels, H.levels)):
        assert_bitwise(host(Ud), Uo, f"level {k}")
    for i in range(2):
        assert bg[i].mass == bo[i].mass and list(bg[i].vel) == list(bo[i].vel)
    assert bo[0].mass > 5.0


def test_nested_coupled_live_orbit_selfgravity(orc, bsn):
    # dt held at the driver's dt_max (below every CFL dt of these steps), so
    # both loops take the same dts and the states differ only by the rounding
    # of the gas-force and FFT sums carried through three steps; with the gas
    # CFL alone the next dt comes from a near-vacuum cell beside a sink where
    # v = m / rho magnifies that rounding
    H, Hd, bo, bg, x0 = _setup(orc, bsn)
    t_ref = _oracle_loop(H, bo, x0, 3, True, True, dt_max=5e-4)
    t, n = bsn.coupled_nested_run_steps(Hd, bg, x0, x0, x0, 0.4, n_steps=3, dt_max=5e-4, f_sink=1.0,
                                        torque_free=True, self_gravity=True, rho_sink_min=2e-8, evolve_orbit=True)
    assert n == 3 and t == t_ref
    # momentum components against the largest momentum component (z momentum
    # alone is tiny in this orbit-plane-symmetric problem).  The problem
    # amplifies rounding: the oracle itself, rerun from a state perturbed by
    # 1e-15 relative, moves by the amount measured here (sens), so the bound
    # is the larger of 1e-10 and 10 x that sensitivity.
    def rel(A, B):
        out = []
        for Ua, Ub in zip(A, B):
            scale = [np.abs(Ub[0]).max()] + [np.abs(Ub[1:4]).max()] * 3 + [np.abs(Ub[4]).max()]
            out.append([float(np.abs(Ua[q] - Ub[q]).max() / scale[q]) for q in range(5)])
        return out
    err = rel([host(Ud) for Ud in Hd.levels], H.levels)
    Hp, _, bp, _, _ = _setup(orc, bsn)
    rng = np.random.default_rng(5)
    for Up in Hp.levels:
        Up[0] *= 1.0 + 1e-15 * rng.standard_normal(Up[0].shape)
    _oracle_loop(Hp, bp, x0, 3, True, True, dt_max=5e-4)
    sens = rel(Hp.levels, H.levels)
    print("GPU vs oracle", err, "oracle vs perturbed oracle", sens)
    bound = max(1e-10, 10 * max(max(s) for s in sens))
    assert max(max(e) for e in err) <= bound, (err, sens)
    for i in range(2):
        assert abs(bg[i].mass - bo[i].mass) <= 1e-13 * bo[i].mass
        assert np.allclose(list(bg[i].pos), list(bo[i].pos), rtol=0, atol=1e-13)


def test_nested_coupled_t_end_diagnostics_and_fp32(orc, bsn):
    H, H64, _, b64, x0 = _setup(orc, bsn)
    _, H32, _, b32, _ = _setup(orc, bsn)
    # one full CFL step, after which the sinks' surroundings limit dt to ~1e-4:
    # five steps in all
    t_end = H.cfl_dt(0.4) + 4e-4
    kw = dict(n_steps=1000, t_end=t_end, f_sink=1.0, rho_sink_min=2e-8, self_gravity=True)
    rec = torch.zeros((8, bsn.DIAG_RECORD), dtype=torch.float64, device="cuda")
    t64, n64 = bsn.coupled_nested_run_steps(H64, b64, x0, x0, x0, 0.4, diag=rec, **kw)
    t32, n32 = bsn.coupled_nested_run_steps(H32, b32, x0, x0, x0, 0.4, precision="f32", **kw)
    assert t64 == t_end and t32 == t_end and n64 >= 3
    R = rec.cpu().numpy()
    n0 = H64.dims[0][0]
    dx0 = 8.0 / n0
    end = bsn.diagnostics(H64.levels[0], n0, n0, n0, dx0, dx0, dx0, x0, x0, x0, b64, 4 / 3)
    assert R[n64 - 1, 0] == t64 and np.array_equal(R[n64 - 1, 2:12], end) and np.all(R[n64:] == 0.0)
    a = (0,) + (slice(NG, -NG),) * 3
    for A, B in zip(H32.levels, H64.levels):
        A, B = host(A)[a], host(B)[a]
        assert np.abs(A - B).sum() / np.abs(B).sum() < 1e-4
