"""The device-resident FMR loop (bsn_fmr3d_run_steps: dt on the device, one
CUDA graph per step, coarse step and first fine subcycle batched into one
launch per RK3 stage) against the reference driver loop on the oracle
(`dt = cfl_dt_fmr3d; dt = min(dt, t_end - t); fmr3d_step!; t += dt`):
equal states (== comparison: the first subcycle reads U_c^n where the
reference forms 1*U_c^n + 0*U_c^{n+1}, which can differ only in the sign of
a zero), the same step count and end time; FP32 and learned stencils close
to FP64."""
import numpy as np
import pytest

from gpu_util import NG, assert_bitwise, dev, host, random_state
from test_gpu_fmr import _pair, _sedov_fmr, _smooth_sg_grid

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


def _reference_loop(Go, cfl, t_end, **kw):
    t, steps = 0.0, 0
    while t < t_end:
        dt = min(Go.cfl_dt(cfl), t_end - t)
        Go.step(dt, **kw)
        t += dt
        steps += 1
    return t, steps


def test_fmr_run_steps_sedov_matches_reference_loop(orc, bsn):
    Go, Gd = _sedov_fmr(orc, bsn)
    t_ref, n_ref = _reference_loop(Go, 0.4, 0.01)
    l0 = bsn.launch_count()
    t, n = bsn.fmr3d_run_steps(Gd, 0.4, n_steps=10000, t_end=0.01)
    assert (t, n) == (t_ref, n_ref)
    assert n >= 2 and bsn.launch_count() > l0
    assert_bitwise(host(Gd.Uc), Go.Uc, "coarse")
    assert_bitwise(host(Gd.Uf), Go.Uf, "fine")


@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_fmr_run_steps_ratio2_random(orc, bsn, bc):
    Uc = random_state(16, 16, 12, seed=33, gamma=5 / 3)
    (orc.fill_ghost_3d_outflow if bc == "outflow" else orc.fill_ghost_3d_periodic)(Uc)
    Go, Gd = _pair(orc, bsn, Uc, 0.0625, (6, 6, 5), (11, 10, 8), 2, 5 / 3, bc=bc, rho_floor=1e-8, P_floor=1e-6)
    t_ref = 0.0
    for _ in range(3):
        dt = Go.cfl_dt(0.3)
        Go.step(dt)
        t_ref += dt
    t, n = bsn.fmr3d_run_steps(Gd, 0.3, n_steps=3)
    assert n == 3 and t == t_ref
    assert_bitwise(host(Gd.Uc), Go.Uc, "coarse")
    assert_bitwise(host(Gd.Uf), Go.Uf, "fine")
    # a second call continues from t (graph reused)
    dt = Go.cfl_dt(0.3)
    Go.step(dt)
    t2, n2 = bsn.fmr3d_run_steps(Gd, 0.3, n_steps=1, t=t)
    assert n2 == 1 and t2 == t + dt
    assert_bitwise(host(Gd.Uc), Go.Uc, "coarse, second call")


def test_fmr_run_steps_selfgravity(orc, bsn):
    Go, Gd = _smooth_sg_grid(orc, bsn)
    for _ in range(2):
        Go.step(Go.cfl_dt(0.4), self_gravity=True, G_grav=0.5)
    t, n = bsn.fmr3d_run_steps(Gd, 0.4, n_steps=2, self_gravity=True, G_grav=0.5)
    assert n == 2
    for A, B in ((host(Gd.Uc), Go.Uc), (host(Gd.Uf), Go.Uf)):
        for q in range(5):
            scale = max(np.abs(B[q]).max(), 1e-300)
            assert np.abs(A[q] - B[q]).max() <= 1e-12 * scale, q


@pytest.mark.parametrize("prec", ["f32", "learned"])
def test_fmr_run_steps_reduced_precision_close_to_fp64(orc, bsn, prec):
    if prec == "learned":
        from bsn import learned as L
        L.install(*L.load_params())
    Go, G64 = _sedov_fmr(orc, bsn)
    _, Gp = _sedov_fmr(orc, bsn)
    t64, n64 = bsn.fmr3d_run_steps(G64, 0.4, n_steps=10000, t_end=0.01)
    tp, npr = bsn.fmr3d_run_steps(Gp, 0.4, n_steps=10000, t_end=0.01, precision=prec)
    assert tp == t64
    tol = 1e-4 if prec == "f32" else 2e-2   # relative L1 of rho on each level
    for A, B in ((host(Gp.Uc), host(G64.Uc)), (host(Gp.Uf), host(G64.Uf))):
        a = (0,) + (slice(NG, -NG),) * 3
        assert np.isfinite(A).all()
        assert np.abs(A[a] - B[a]).sum() / np.abs(B[a]).sum() < tol


def test_fmr_run_steps_selfgravity_fp32_transforms(orc, bsn):
    """FP32 stencils and FP32 FFTs with self-gravity stay close to the FP64 loop."""
    _, G64 = _smooth_sg_grid(orc, bsn)
    _, G32 = _smooth_sg_grid(orc, bsn)
    t64, _ = bsn.fmr3d_run_steps(G64, 0.4, n_steps=3, self_gravity=True)
    t32, _ = bsn.fmr3d_run_steps(G32, 0.4, n_steps=3, self_gravity=True, precision="f32")
    assert abs(t32 - t64) <= 1e-6 * t64
    a = (0,) + (slice(NG, -NG),) * 3
    for A, B in ((host(G32.Uc), host(G64.Uc)), (host(G32.Uf), host(G64.Uf))):
        assert np.abs(A[a] - B[a]).sum() / np.abs(B[a]).sum() < 1e-5
