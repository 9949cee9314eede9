"""TMA staging of the fused stage kernel (csrc/tma.cuh, csrc/stage_tile.cuh
stage_cross_tma): the block and its halos copied into shared memory by
cp.async.bulk.tensor in chunks, converted from there.

The FP64 path through the TMA kernel must stay bit-identical to the oracle
(src/euler3d.jl:220-260) for every tile variant and both boundary
conditions, including the boundary blocks whose out-of-domain halo cells come
through the boundary map.  The FP32 path must give the same bits with TMA
staging as with the plain per-thread loader (same arithmetic on the same
staged values); the learned stage's screening launch keeps the plain loader.  Profiling records show that the TMA kernels
ran, and grids the copies cannot describe (odd nx, a tile not dividing the
grid) fall back to the plain loader.
"""
import numpy as np
import pytest

from gpu_util import assert_bitwise, dev, host, random_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    yield b
    b.set_tma(True)
    for p in ("f64", "f32", "learned"):
        b.set_tile(p, -1)


def _step_counts(bsn, step, U, n, d, dt, name):
    bsn.set_profiling(True)
    step(U, *n, *d, dt, 5 / 3, rho_floor=1e-6, P_floor=1e-6)
    torch.cuda.synchronize()
    cnt = bsn.kernel_time(name)[1]
    bsn.set_profiling(False)
    return cnt


@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_fp64_tma_steps_bitwise_every_tile(orc, bsn, bc):
    n, d = (32, 16, 16), (0.05, 0.07, 0.06)
    U0 = random_state(*n, seed=81, gamma=5 / 3, vacuum=True)
    bsn.set_tma(True)
    for v in range(bsn.tile_variants("f64")):
        bsn.set_tile("f64", v)
        U = U0.copy(order="F")
        Ud = dev(U)
        for _ in range(2):
            dt = 2e-3
            orc.euler3d_step(U, *d, dt, 5 / 3, bc=bc, rho_floor=1e-6, P_floor=1e-6)
            bsn.set_profiling(True)
            bsn.euler3d_step(Ud, *n, *d, dt, 5 / 3, bc=bc, rho_floor=1e-6, P_floor=1e-6)
            torch.cuda.synchronize()
            assert bsn.kernel_time("stage_kernel_tma")[1] == 3, v
            bsn.set_profiling(False)
        assert_bitwise(host(Ud), U, f"FP64 TMA step, tile {v}, {bc}")
    bsn.set_tile("f64", -1)


@pytest.mark.parametrize("path", ["f32"])
def test_reduced_precision_tma_equals_plain_loader(bsn, path):
    step = {"f32": bsn.euler3d_step_f32}[path]
    name = {"f32": "stage_kernel_f32_tma"}[path]
    n, d, dt = (32, 32, 16), (0.05, 0.05, 0.05), 2e-3
    U0 = random_state(*n, seed=83, gamma=5 / 3, vacuum=True)
    for v in range(bsn.tile_variants(path)):
        bsn.set_tile(path, v)
        out = []
        for tma in (True, False):
            bsn.set_tma(tma)
            Ud = dev(U0.copy(order="F"))
            cnt = _step_counts(bsn, step, Ud, n, d, dt, name)
            assert cnt == (3 if tma else 0), (v, tma, cnt)
            step(Ud, *n, *d, dt, 5 / 3, rho_floor=1e-6, P_floor=1e-6)
            out.append(host(Ud))
        assert_bitwise(out[0], out[1], f"{path} TMA vs plain loader, tile {v}")
    bsn.set_tma(True)
    bsn.set_tile(path, -1)


def test_tma_falls_back_where_copies_do_not_apply(orc, bsn):
    # odd nx (row stride not a multiple of 16 bytes) and a tile that does not
    # divide the grid: the plain loader runs, still bit-identical
    bsn.set_tma(True)
    for n in ((17, 16, 16), (24, 12, 20)):
        U = random_state(*n, seed=85, gamma=1.4)
        Ud = dev(U)
        bsn.set_profiling(True)
        bsn.euler3d_step(Ud, *n, 0.1, 0.1, 0.1, 1e-3, 1.4)
        torch.cuda.synchronize()
        tma_launches = bsn.kernel_time("stage_kernel_tma")[1]
        bsn.set_profiling(False)
        orc.euler3d_step(U, 0.1, 0.1, 0.1, 1e-3, 1.4)
        assert_bitwise(host(Ud), U, f"fallback {n}")
        tile = bsn.get_tile(*n, "f64")
        divides = all(a % t == 0 for a, t in zip(n, tile[:3])) and n[0] % 2 == 0
        assert not divides and bsn.get_tile_tma(*n, "f64") is False and tma_launches == 0, (n, tile, tma_launches)


def test_device_loop_with_tma_matches_oracle_loop(orc, bsn):
    # the graph-captured time loop (the bench's path) with TMA staging
    n, dx = 32, 2.0 / 32
    U = orc.state(n, n, n)
    orc.sedov_ic_3d(U, dx, dx, dx, 5 / 3, E_blast=1.0, r_inject=3.5 * dx, rho_bg=1.0, P_floor=1e-5,
                    x_offset=-1.0, y_offset=-1.0, z_offset=-1.0)
    Ud = dev(U)
    bsn.set_tma(True)
    bsn.set_tile("f64", bsn.tile_variants("f64") - 1)   # a forced tile is TMA-staged wherever possible
    t, k = bsn.run_steps(Ud, n, n, n, dx, dx, dx, 5 / 3, 0.4, n_steps=5, precision="f64", rho_floor=1e-6,
                         P_floor=1e-6)
    assert bsn.get_tile_tma(n, n, n, "f64") is True
    bsn.set_tile("f64", -1)
    assert k == 5
    t_ref = 0.0
    for _ in range(5):
        dt = orc.cfl_dt_3d(U, dx, dx, dx, 5 / 3, 0.4)
        orc.euler3d_step(U, dx, dx, dx, dt, 5 / 3, rho_floor=1e-6, P_floor=1e-6)
        t_ref += dt
    assert t == t_ref
    assert_bitwise(host(Ud), U, "device loop with TMA")


@pytest.mark.parametrize("path", ["f32", "learned"])
def test_every_reduced_precision_tile_variant_gives_the_same_bits(bsn, path):
    """The FP32 stencil units write every multiply-add out and are built
    without contraction, so the autotuner's tile choice cannot change a
    result: two steps with every tile variant, TMA staging on, are
    bit-identical."""
    from bsn import learned as Lw
    if path == "learned":
        Lw.install(*Lw.load_params())
    step = {"f32": bsn.euler3d_step_f32, "learned": bsn.euler3d_step_learned}[path]
    n, d, dt = (32, 32, 16), (0.05, 0.05, 0.05), 2e-3
    U0 = random_state(*n, seed=87, gamma=5 / 3, vacuum=True)
    bsn.set_tma(True)
    outs = []
    for v in range(bsn.tile_variants(path)):
        bsn.set_tile(path, v)
        Ud = dev(U0.copy(order="F"))
        for _ in range(2):
            step(Ud, *n, *d, dt, 5 / 3, rho_floor=1e-6, P_floor=1e-6)
        outs.append(host(Ud))
    bsn.set_tile(path, -1)
    for v in range(1, len(outs)):
        assert_bitwise(outs[v], outs[0], f"{path} tile {v} vs tile 0")
