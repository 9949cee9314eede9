"""Nested FMR on the device (bsn_fmr_nested_step_f64, bsn_cfl_dt_fmr_nested_f64,
bsn_fmr_nested_run_steps) against the oracle's recursive restatement of
fmr3d_step! (src/fmr3d.jl:451-604 with every level subcycling inside its
parent; src/fmr_gravity.jl pair by pair for self-gravity).  Hydro steps are
compared with == (the first substep of a chain reads its parent's saved state
where the oracle forms 1*U^n + 0*U^{n+1}, which can differ only in the sign
of a zero); steps with self-gravity within 1e-12 (the FFT)."""
import numpy as np
import pytest

from gpu_util import NG, assert_bitwise, dev, host, random_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


def _nested(orc, bsn, U0, dx0, boxes, gamma, **kw):
    Ho = orc.FMRHierarchy(U0.copy(order="F"), dx0, boxes, gamma, **kw)
    Hd = bsn.FMRHierarchy3D(dev(U0), *orc.dims(U0), dx0, boxes, gamma, **kw)
    return Ho, Hd


def _set_levels(orc, Ho, Hd, dx0, L, boxes, fill):
    """Give every finer level its own analytic state fill(U, dx, x0), ghosts
    from its parent, and copy the oracle's levels to the device."""
    x0, dx = -L, dx0
    for k, b in enumerate(boxes):
        x0 = x0 + (b[0] - 1) * dx
        dx = dx / b[6]
        fill(Ho.levels[k + 1], dx, x0)
        Ho.pairs[k].prolong_fine_ghosts()
    for Ud, Uo in zip(Hd.levels, Ho.levels):
        Ud.copy_(dev(Uo))


SEDOV_BOXES = ((5, 12, 5, 12, 5, 12, 2), (5, 12, 5, 12, 5, 12, 2))


def _sedov3(orc, bsn, nc=16, L=0.5, boxes=SEDOV_BOXES, g=5 / 3):
    dx0 = 2 * L / nc
    U0 = orc.state(nc, nc, nc)

    def fill(U, dx, x0):
        orc.sedov_ic_3d(U, dx, dx, dx, g, E_blast=1.0, r_inject=0.15, rho_bg=1.0, P_floor=1e-5,
                        x_offset=x0, y_offset=x0, z_offset=x0)

    fill(U0, dx0, -L)
    orc.fill_ghost_3d_outflow(U0)
    Ho, Hd = _nested(orc, bsn, U0, dx0, boxes, g, rho_floor=1e-10, P_floor=1e-5)
    _set_levels(orc, Ho, Hd, dx0, L, boxes, fill)
    return Ho, Hd


def _blob3(orc, bsn, nc=16, L=0.5, boxes=SEDOV_BOXES, sigma=0.15, g=5 / 3):
    # smooth self-gravitating Gaussian (no prolongation overshoot to rho <= 0)
    dx0 = 2 * L / nc

    def fill(U, dx, x0):
        n = U.shape[1] - 2 * NG
        c = (np.arange(n) + 0.5) * dx + x0
        X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
        rho = 1e-2 + np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / (2 * sigma ** 2))
        a = (slice(NG, NG + n),) * 3
        U[(0,) + a] = rho
        U[(4,) + a] = rho * 1e-2

    U0 = orc.state(nc, nc, nc)
    fill(U0, dx0, -L)
    orc.fill_ghost_3d_outflow(U0)
    Ho, Hd = _nested(orc, bsn, U0, dx0, boxes, g, rho_floor=1e-12, P_floor=1e-12)
    _set_levels(orc, Ho, Hd, dx0, L, boxes, fill)
    return Ho, Hd


def _levels_bitwise(Ho, Hd, what):
    for k, (Uo, Ud) in enumerate(zip(Ho.levels, Hd.levels)):
        assert_bitwise(host(Ud), Uo, f"{what}, level {k}")


def _levels_close(Ho, Hd, tol):
    for k, (Uo, Ud) in enumerate(zip(Ho.levels, Hd.levels)):
        A = host(Ud)
        for q in range(5):
            scale = max(np.abs(Uo[q]).max(), 1e-300)
            assert np.abs(A[q] - Uo[q]).max() <= tol * scale, (k, q)


def test_nested_prolong_all_matches_oracle(orc, bsn):
    U0 = random_state(16, 16, 12, seed=41, gamma=5 / 3)
    orc.fill_ghost_3d_outflow(U0)
    boxes = ((6, 11, 6, 10, 5, 8, 2), (4, 9, 4, 7, 3, 6, 2))
    Ho, Hd = _nested(orc, bsn, U0, 0.0625, boxes, 5 / 3)
    _levels_bitwise(Ho, Hd, "prolong_all")


def test_two_level_nested_equals_fmr3d_step(orc, bsn):
    from test_gpu_fmr import _sedov_fmr
    _, G = _sedov_fmr(orc, bsn)
    _, G2 = _sedov_fmr(orc, bsn)
    H = bsn.FMRHierarchy3D.__new__(bsn.FMRHierarchy3D)
    H.pairs, H.levels = [G2], [G2.Uc, G2.Uf]
    H._arr = (bsn.api.bsn_fmr2 * 1)(G2.s)
    for _ in range(3):
        dt = bsn.cfl_dt_fmr3d(G, 0.4)
        assert bsn.cfl_dt_fmr_nested(H, 0.4) == dt
        bsn.fmr3d_step(G, dt)
        bsn.fmr_nested_step(H, dt)
    assert torch.equal(G.Uc, G2.Uc) and torch.equal(G.Uf, G2.Uf)


@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_three_level_random_steps_bitwise(orc, bsn, bc):
    U0 = random_state(16, 16, 12, seed=42, gamma=5 / 3)
    (orc.fill_ghost_3d_outflow if bc == "outflow" else orc.fill_ghost_3d_periodic)(U0)
    boxes = ((6, 11, 6, 10, 5, 8, 2), (4, 9, 4, 7, 3, 6, 2))
    Ho, Hd = _nested(orc, bsn, U0, 0.0625, boxes, 5 / 3, bc=bc, rho_floor=1e-8, P_floor=1e-6)
    for step in range(3):
        dt = Ho.cfl_dt(0.3)
        assert bsn.cfl_dt_fmr_nested(Hd, 0.3) == dt
        Ho.step(dt)
        bsn.fmr_nested_step(Hd, dt)
        _levels_bitwise(Ho, Hd, f"step {step}")


def test_three_level_ratio4_and_2(orc, bsn):
    U0 = random_state(12, 12, 12, seed=43, gamma=1.4, jumps=False)
    orc.fill_ghost_3d_outflow(U0)
    boxes = ((5, 8, 5, 8, 5, 8, 4), (5, 12, 6, 11, 5, 12, 2))
    Ho, Hd = _nested(orc, bsn, U0, 1 / 12, boxes, 1.4, rho_floor=1e-8, P_floor=1e-6)
    for _ in range(2):
        dt = Ho.cfl_dt(0.4)
        Ho.step(dt)
        bsn.fmr_nested_step(Hd, dt)
    _levels_bitwise(Ho, Hd, "ratios 4, 2")


def test_three_level_sedov_run_matches_reference_loop(orc, bsn):
    Ho, Hd = _sedov3(orc, bsn)
    t_ref, n_ref = 0.0, 0
    while t_ref < 0.01:
        dt = min(Ho.cfl_dt(0.4), 0.01 - t_ref)
        Ho.step(dt)
        t_ref += dt
        n_ref += 1
    l0 = bsn.launch_count()
    t, n = bsn.fmr_nested_run_steps(Hd, 0.4, n_steps=10000, t_end=0.01)
    assert (t, n) == (t_ref, n_ref) and n >= 2
    assert bsn.launch_count() > l0
    _levels_bitwise(Ho, Hd, "sedov run")
    # a second call continues from t (graph reused)
    dt = Ho.cfl_dt(0.4)
    Ho.step(dt)
    t2, n2 = bsn.fmr_nested_run_steps(Hd, 0.4, n_steps=1, t=t)
    assert n2 == 1 and t2 == t + dt
    _levels_bitwise(Ho, Hd, "second call")


@pytest.mark.parametrize("G_grav", [1.0, 0.5])
def test_three_level_selfgravity_matches_oracle(orc, bsn, G_grav):
    Ho, Hd = _blob3(orc, bsn)
    for _ in range(2):
        dt = Ho.cfl_dt(0.4)
        Ho.step(dt, self_gravity=True, G_grav=G_grav)
        bsn.fmr_nested_step(Hd, dt, self_gravity=True, G_grav=G_grav)
    _levels_close(Ho, Hd, 1e-12)


def test_three_level_selfgravity_run(orc, bsn):
    Ho, Hd = _blob3(orc, bsn)
    for _ in range(2):
        Ho.step(Ho.cfl_dt(0.4), self_gravity=True, G_grav=0.5)
    t, n = bsn.fmr_nested_run_steps(Hd, 0.4, n_steps=2, self_gravity=True, G_grav=0.5)
    assert n == 2
    _levels_close(Ho, Hd, 1e-12)


@pytest.mark.parametrize("prec", ["f32", "learned"])
def test_three_level_reduced_precision_close_to_fp64(orc, bsn, prec):
    if prec == "learned":
        from bsn import learned as Lm
        Lm.install(*Lm.load_params())
    _, H64 = _sedov3(orc, bsn)
    _, Hp = _sedov3(orc, bsn)
    t64, n64 = bsn.fmr_nested_run_steps(H64, 0.4, n_steps=10000, t_end=0.01)
    tp, npr = bsn.fmr_nested_run_steps(Hp, 0.4, n_steps=10000, t_end=0.01, precision=prec)
    assert tp == t64
    # relative L1 of rho on each level; the finest level takes four substeps
    # per level-0 step inside the blast, where FP32 rounding grows fastest
    tol = 3e-4 if prec == "f32" else 2e-2
    a = (0,) + (slice(NG, -NG),) * 3
    errs = []
    for A, B in zip(Hp.levels, H64.levels):
        A, B = host(A), host(B)
        assert np.isfinite(A).all()
        errs.append(np.abs(A[a] - B[a]).sum() / np.abs(B[a]).sum())
    assert max(errs) < tol, errs


def test_broken_chain_is_rejected(orc, bsn):
    _, Hd = _sedov3(orc, bsn)
    arr = (bsn.api.bsn_fmr2 * 2)(*[p.s for p in Hd.pairs])
    arr[1].Uc = Hd.levels[0].data_ptr()
    with pytest.raises(bsn.BSNError, match="not pair"):
        bsn.api._call("bsn_fmr_nested_step_f64", bsn.context(), arr, 2, 1e-4, 0, 1.0)
