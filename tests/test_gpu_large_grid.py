"""The uniform-grid step on a grid whose state array holds more than 2^31
doubles (760^3 active cells: 766^3 x 5 = 2.25e9 elements, 18 GB per array),
so every offset past z-plane ~732 needs 64-bit arithmetic.

The grid is a uniform flow with a random blob (shock and near-vacuum cells
included) in its far corner.  A step only reads nine cells around each cell,
so the corner's 24^3 active cells must come out exactly as the oracle's step
(src/euler3d.jl:220-260) of a 24^3 grid holding the same corner; the CFL
maximum over 4.4e8 cells must equal the small grid's.  Needs ~80 GB free on
the device (the state, two stage buffers and the autotuner's scratch)."""
import numpy as np
import pytest

from gpu_util import NG, dev, host

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N = 760          # large grid, active cells per axis
M = 24           # the corner copied into a small grid
BG = (1.0, 0.1, -0.2, 0.05, 2.5 + 0.5 * (0.01 + 0.04 + 0.0025))   # rho, momenta, E (P = 1, gamma = 1.4)
KW = dict(rho_floor=1e-6, P_floor=1e-5)


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


def _small(orc, seed=11):
    """M^3 grid: the uniform background with a random blob in its last 10
    active cells along every axis, outflow ghosts."""
    rng = np.random.default_rng(seed)
    S = orc.state(M, M, M)
    for q in range(5):
        S[q] = BG[q]
    c = (slice(NG + M - 10, NG + M),) * 3
    rho = np.abs(1.0 + 0.5 * rng.standard_normal((10, 10, 10))) + 0.05
    rho[:5] *= 8.0                                   # a density jump
    rho[rng.random((10, 10, 10)) < 0.03] = 1e-9      # near-vacuum cells (floors)
    v = 0.8 * rng.standard_normal((3, 10, 10, 10))
    P = np.abs(1.0 + 0.4 * rng.standard_normal((10, 10, 10))) + 0.01
    P[:, :4] *= 50.0                                 # a pressure jump
    S[(0,) + c] = rho
    S[(slice(1, 4),) + c] = rho * v
    S[(4,) + c] = P / 0.4 + 0.5 * rho * (v ** 2).sum(0)
    orc.fill_ghost_3d_outflow(S)
    return S


def _large(bsn, S):
    """The N^3 device grid: background everywhere, S in the far corner
    (ghosts included: outflow copies of the same cells)."""
    U = bsn.state(N, N, N)
    for q in range(5):
        U[q].fill_(BG[q])
    w = M + 2 * NG
    U[:, -w:, -w:, -w:] = dev(S)
    return U


def _corner(U):
    """The corner's active cells as the small grid indexes them."""
    w = M + 2 * NG
    return host(U[:, -w:, -w:, -w:].contiguous())[:, NG:-NG, NG:-NG, NG:-NG]


@pytest.fixture(scope="module")
def room():
    free, _ = torch.cuda.mem_get_info()
    need = 4 * 5 * (N + 2 * NG) ** 3 * 8 + (4 << 30)
    if free < need:
        pytest.skip(f"{need / 1e9:.0f} GB of device memory needed, {free / 1e9:.0f} GB free")
    assert 5 * (N + 2 * NG) ** 3 > 2 ** 31
    yield
    torch.cuda.empty_cache()


def test_large_grid_fp64_step_and_cfl_bitwise(orc, bsn, room):
    g, dx = 1.4, 1.0 / N
    S = _small(orc)
    U = _large(bsn, S)
    dt = bsn.cfl_dt_3d(U, N, N, N, dx, dx, dx, g, 0.4)
    assert dt == orc.cfl_dt_3d(S, dx, dx, dx, g, 0.4)
    bsn.euler3d_step(U, N, N, N, dx, dx, dx, dt, g, **KW)
    orc.euler3d_step(S, dx, dx, dx, dt, g, **KW)
    got = _corner(U)
    want = S[:, NG:-NG, NG:-NG, NG:-NG]
    assert np.array_equal(got, want), int((got != want).sum())
    # the device time loop (device-resident dt, graph-captured step) on a fresh grid
    S2 = _small(orc)
    U = _large(bsn, S2)
    t, n = bsn.run_steps(U, N, N, N, dx, dx, dx, g, 0.4, n_steps=1, **KW)
    orc.euler3d_step(S2, dx, dx, dx, dt, g, **KW)
    assert (t, n) == (dt, 1)
    assert np.array_equal(_corner(U), S2[:, NG:-NG, NG:-NG, NG:-NG])


@pytest.mark.parametrize("prec", ["f32", "learned"])
def test_large_grid_reduced_precision_step(orc, bsn, room, prec):
    g, dx = 1.4, 1.0 / N
    if prec == "learned":
        from bsn import learned
        learned.install(*learned.load_params())
    step = bsn.euler3d_step_f32 if prec == "f32" else bsn.euler3d_step_learned
    S = _small(orc)
    dt = orc.cfl_dt_3d(S, dx, dx, dx, g, 0.4)
    # one tile variant for both grids (each variant is compiled on its own, so
    # two variants may contract multiply-adds differently); every variant's
    # tile sizes divide N - M, so the corner's blocks hold the same cells
    bsn.set_tile(prec, 0)
    try:
        U = _large(bsn, S)
        step(U, N, N, N, dx, dx, dx, dt, g, **KW)
        V = dev(S)
        step(V, M, M, M, dx, dx, dx, dt, g, **KW)
    finally:
        bsn.set_tile(prec, -1)
    got, small = _corner(U), host(V)[:, NG:-NG, NG:-NG, NG:-NG]
    orc.euler3d_step(S, dx, dx, dx, dt, g, **KW)
    want = S[:, NG:-NG, NG:-NG, NG:-NG]
    assert np.isfinite(got).all()
    # the same cells through the small grid: the arithmetic of a cell does not
    # depend on the grid size or where the cell sits in memory
    if not np.array_equal(got, small):
        d = got != small
        rel = np.max(np.abs(got - small)[d] / np.maximum(np.abs(small[d]), 1e-300))
        raise AssertionError(f"{int(d.sum())} values differ from the small grid's (max rel {rel:.2e}) at "
                             f"{np.argwhere(d)[:4].tolist()}")
    # and within the reduced-precision tolerance of the FP64 oracle step
    tol = 1e-5 if prec == "f32" else 1e-3
    for q in (0, 4):
        err = np.abs(got[q] - want[q]).sum() / np.abs(want[q]).sum()
        assert err < tol, (q, err)
