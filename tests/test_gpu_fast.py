"""GPU tests of the tile autotuner, the graph-captured device time loop and
the FP32-stencil fast path.

* Every FP64 tile variant gives bit-identical results (the tiling changes
  only which CTA computes an interface, never the arithmetic).
* bsn_run_steps (dt, t and the CFL maximum on the device, one CUDA graph per
  step) reproduces the reference driver loop `dt = cfl_dt_3d; dt = min(dt,
  t_end - t); euler3d_step!; t += dt` bit for bit, including the step count.
* The FP32 path (FP32 stencils, FP64 state) stays within a stated L1 distance
  of the FP64 oracle: L1(rho) and L1(E) relative below 1e-5 on Sedov 32^3 to
  t = 0.1 and on one random-state step.
"""
import numpy as np
import torch
import pytest

from gpu_util import NG, assert_bitwise, dev, host, random_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


def _sedov(orc, n=32, L=1.0, g=5 / 3):
    dx = 2 * L / n
    U = orc.state(n, n, n)
    orc.sedov_ic_3d(U, dx, dx, dx, g, E_blast=1.0, r_inject=3.5 * dx, rho_bg=1.0, P_floor=1e-5,
                    x_offset=-L, y_offset=-L, z_offset=-L)
    return U, dx


def test_every_fp64_tile_variant_is_bitwise(orc, bsn):
    n = (37, 21, 19)
    U = random_state(*n, seed=41, vacuum=True)
    ref = U.copy(order="F")
    orc.euler3d_step(ref, 0.1, 0.07, 0.13, 2e-3, 1.4, rho_floor=1e-6, P_floor=1e-4)
    try:
        for v in range(bsn.tile_variants("f64")):
            bsn.set_tile("f64", v)
            Ud = dev(U)
            bsn.euler3d_step(Ud, *n, 0.1, 0.07, 0.13, 2e-3, 1.4, rho_floor=1e-6, P_floor=1e-4)
            assert_bitwise(host(Ud), ref, f"tile variant {v}")
    finally:
        bsn.set_tile("f64", -1)


def test_autotuner_picks_a_variant(bsn):
    U = bsn.state(40, 40, 40)
    U[0] = 1.0
    U[4] = 2.5
    bsn.euler3d_step(U, 40, 40, 40, 0.1, 0.1, 0.1, 1e-3, 1.4)
    tx, ty, tz, nt, minb = bsn.get_tile(40, 40, 40, "f64")
    assert tx * ty * tz % nt == 0 and nt in (128, 256, 512)


@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_run_steps_f64_matches_reference_loop(orc, bsn, bc):
    U, dx = _sedov(orc)
    Ud = dev(U)
    g, tend = 5 / 3, 0.02
    t, steps = 0.0, 0
    while t < tend:
        dt = min(orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4), tend - t)
        orc.euler3d_step(U, dx, dx, dx, dt, g, bc=bc, rho_floor=1e-6, P_floor=1e-6)
        t += dt
        steps += 1
    # more graph launches than needed: the loop must stop at t_end by itself
    tg, ng = bsn.run_steps(Ud, 32, 32, 32, dx, dx, dx, g, 0.4, n_steps=steps + 5, t=0.0, t_end=tend, bc=bc,
                           rho_floor=1e-6, P_floor=1e-6, precision="f64")
    assert ng == steps and tg == t
    assert_bitwise(host(Ud), U, "run_steps end state")


def test_run_steps_fixed_count_and_resume(orc, bsn):
    U, dx = _sedov(orc, n=24)
    Ud = dev(U)
    g = 5 / 3
    t = 0.0
    for _ in range(4):
        dt = orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4)
        orc.euler3d_step(U, dx, dx, dx, dt, g, rho_floor=1e-6, P_floor=1e-6)
        t += dt
    t1, n1 = bsn.run_steps(Ud, 24, 24, 24, dx, dx, dx, g, 0.4, n_steps=2, rho_floor=1e-6, P_floor=1e-6)
    t2, n2 = bsn.run_steps(Ud, 24, 24, 24, dx, dx, dx, g, 0.4, n_steps=2, t=t1, rho_floor=1e-6, P_floor=1e-6)
    assert (n1, n2) == (2, 2) and t2 == t
    assert_bitwise(host(Ud), U, "resumed run")


def _l1_rel(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


def test_fp32_step_close_to_fp64(orc, bsn):
    # random states with jumps: the FP32 WENO-Z weights of stencils beside a
    # jump (beta ~ 0) dominate the error, so one seed's figure is noisy; the
    # mean over eight seeds is the measure (about 2e-6 for rho and 3e-6 for E)
    n = (24, 20, 16)
    a = (slice(NG, -NG),) * 3
    err = []
    for seed in range(40, 48):
        U = random_state(*n, seed=seed)
        ref = U.copy(order="F")
        orc.euler3d_step(ref, 0.1, 0.1, 0.1, 1e-3, 1.4, rho_floor=1e-6, P_floor=1e-4)
        Ud = dev(U)
        bsn.euler3d_step_f32(Ud, *n, 0.1, 0.1, 0.1, 1e-3, 1.4, rho_floor=1e-6, P_floor=1e-4)
        G = host(Ud)
        err.append([_l1_rel(G[(q,) + a], ref[(q,) + a]) for q in (0, 4)])
    err = np.array(err)
    assert err.mean(0).max() < 1e-5 and err.max() < 3e-5, err


def test_fp32_sedov_run_l1_vs_fp64(orc, bsn):
    U, dx = _sedov(orc)
    Ud = dev(U)
    g, tend = 5 / 3, 0.1
    t = 0.0
    while t < tend:
        dt = min(orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4), tend - t)
        orc.euler3d_step(U, dx, dx, dx, dt, g, rho_floor=1e-6, P_floor=1e-6)
        t += dt
    tg, ng = bsn.run_steps(Ud, 32, 32, 32, dx, dx, dx, g, 0.4, n_steps=10000, t_end=tend, rho_floor=1e-6,
                           P_floor=1e-6, precision="f32")
    assert abs(tg - tend) < 1e-12
    G = host(Ud)
    a = (slice(NG, -NG),) * 3
    e_rho = _l1_rel(G[(0,) + a], U[(0,) + a])
    e_E = _l1_rel(G[(4,) + a], U[(4,) + a])
    print(f"FP32 vs FP64 Sedov 32^3 t=0.1: L1 rho {e_rho:.3e}, L1 E {e_E:.3e}, steps {ng}")
    assert e_rho < 1e-5 and e_E < 1e-5


@pytest.mark.parametrize("dims", [(32, 32, 32), (64, 32, 16)])
def test_poisson_fp32_transforms_close_to_fp64(bsn, dims):
    """The FP32-transform solve (precision form of the FFTs) against the FP64
    solve (itself checked against the oracle to 1e-12): max |dPhi| within
    1e-5 of max |Phi| on a random positive density."""
    nx, ny, nz = dims
    rng = np.random.default_rng(41)
    rho = torch.from_numpy(np.asfortranarray(rng.uniform(0.1, 2.0, (nx, ny, nz)))).cuda()
    h = 1.0 / nx
    p64 = bsn.solve_poisson_isolated(rho, nx, ny, nz, h, h, h)
    p32 = bsn.solve_poisson_isolated(rho, nx, ny, nz, h, h, h, precision="f32")
    err = (p32 - p64).abs().max().item() / p64.abs().max().item()
    assert 0 < err < 1e-5, err


def test_fp32_step_takes_fp64_fluxes_at_stiff_faces(orc, bsn):
    """Faces whose six-cell density stencil spans more than three decades are
    computed in FP64 by the FP32 path when the stiff guard is on (FP32
    rounding of the dense side's values would be 1e-4 and more of the thin
    cell's).  On a 3-D checkerboard of O(1) and 1e-4 densities every face of
    every axis is stiff, so the guarded FP32 face fluxes are the FP64 fluxes
    rounded to FP32 (relative error <= 2^-24 per face, 1e-7 of the axis's
    largest flux taken here), while unguarded FP32 stencils miss them by far
    more.  Fluxes rather than a step are compared: the checkerboard's step
    switches WENO/HLLC branches on 1e-12 perturbations, so its increments
    are not a conditioned measure of the face arithmetic."""
    n, d, g = (16, 16, 16), (0.05, 0.05, 0.05), 5 / 3
    U = random_state(*n, seed=91, gamma=g, jumps=False)
    a = (slice(3, -3),) * 3
    i, j, k = np.meshgrid(*(np.arange(m) for m in n), indexing="ij")
    scale = np.where((i + j + k) % 2 == 1, 1e-4, 1.0)
    for q in range(5):
        U[(q,) + a] = U[(q,) + a] * scale
    orc.fill_ghost_3d_outflow(U)
    flux = {}
    for name, guard in (("f64", None), ("guarded", True), ("plain", False)):
        Ud = dev(U)
        dUd = torch.zeros_like(Ud)
        F = [torch.zeros_like(dev(f)) for f in orc.flux_arrays(*n)]
        if guard is None:
            bsn.euler3d_rhs(dUd, *F, Ud, *n, *d, g, rho_floor=1e-10, P_floor=1e-14)
        else:
            bsn.set_stiff_guard(guard)
            try:
                bsn.euler3d_rhs_f32(dUd, *F, Ud, *n, *d, g, rho_floor=1e-10, P_floor=1e-14)
            finally:
                bsn.set_stiff_guard(False)
        flux[name] = [host(f) for f in F]
    err = {}
    for name in ("guarded", "plain"):
        err[name] = max(float(np.abs(f - r)[q].max() / np.abs(r[q]).max())
                        for f, r in zip(flux[name], flux["f64"]) for q in range(5))
    print("face fluxes vs FP64, max relative: guarded %.2e, plain FP32 %.2e" % (err["guarded"], err["plain"]))
    assert err["guarded"] < 1e-7, err
    assert err["plain"] > 100 * err["guarded"], err
