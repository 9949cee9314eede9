"""The z-slab step (bsn/shard.py) with the library's device operations on one
GPU: a single rank holding the whole grid is bit-identical to the oracle's
euler3d_step! driver loop (the halo logic itself is checked across gloo ranks
in test_shard.py), and the flooring of received halo planes equals the
oracle's apply_floors_3d! on those planes."""
import numpy as np
import pytest

from gpu_util import NG, assert_bitwise, dev, host, random_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("bc", ["outflow", "periodic"])
def test_single_slab_matches_oracle_loop(orc, bc):
    from bsn import shard
    n, nz, dx, g = 12, 10, 0.1, 1.4
    kw = dict(rho_floor=1e-6, P_floor=1e-5)
    U = random_state(n, n, nz, seed=11, vacuum=True)
    (orc.fill_ghost_3d_outflow if bc == "outflow" else orc.fill_ghost_3d_periodic)(U)
    Ud = dev(U)
    slab = shard.Slab.split(n, n, nz, 0, 1, bc)
    t, steps = shard.run_steps(Ud, slab, dx, dx, dx, g, 0.4, shard.DeviceOps(), n_steps=3, **kw)
    t_ref = 0.0
    for _ in range(3):
        dt = orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4)
        orc.euler3d_step(U, dx, dx, dx, dt, g, bc=bc, **kw)
        t_ref += dt
    assert (t, steps) == (t_ref, 3)
    assert_bitwise(host(Ud), U, "single slab")


def test_halo_planes_are_floored_like_the_oracle(orc):
    from bsn import shard
    n = 9
    P = random_state(n, n, NG, seed=12, vacuum=True)
    planes = torch.from_numpy(P.T)[NG:2 * NG].clone().cuda()
    got = shard.DeviceOps().floor_planes(planes, n, n, 1e-6, 1e-5, 1.4).cpu().numpy()
    orc.apply_floors_3d(P, 1e-6, 1e-5, 1.4)
    want = P.T[NG:2 * NG]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_slab_poisson_bitwise_to_the_undivided_solve(orc, world):
    """The distributed isolated Poisson solve, its ranks emulated one after
    another in one process (the all-to-alls done by hand), assembles the
    undivided bsn_solve_poisson_isolated_f64 potential bit for bit; that one
    is within 1e-12 of the oracle."""
    import bsn
    from bsn import shard
    nx, ny, nz, d = 32, 16, 64, (0.05, 0.07, 0.03)
    rng = np.random.default_rng(3)
    rho_h = np.asfortranarray(np.abs(rng.standard_normal((nx, ny, nz))) + 0.1)
    rho = dev(rho_h)
    ref = bsn.solve_poisson_isolated(rho, nx, ny, nz, *d)
    want = orc.solve_poisson_isolated(rho_h, *d)
    assert np.abs(host(ref) - want).max() <= 1e-12 * np.abs(want).max()
    ops = shard.DeviceOps()
    P = [shard.SlabPoisson(shard.Slab.split(nx, ny, nz, r, world), *d, ops) for r in range(world)]
    nzl = nz // world
    sent = [P[r].forward(rho[:, :, r * nzl:(r + 1) * nzl]) for r in range(world)]
    lines = [P[r].lines([sent[s][r] for s in range(world)]) for r in range(world)]
    phi = [P[r].inverse([lines[s][r] for s in range(world)]) for r in range(world)]
    got = torch.cat(phi, 2)
    assert torch.equal(got, ref)


@pytest.mark.parametrize("world", [2, 4])
def test_slab_self_gravity_source_bitwise(orc, world):
    """The self-gravity source on slabs (distributed Phi, one plane of Phi from
    each neighbour, the gradient taking those planes at the slab's edges), ranks
    emulated one after another in one process: bit-identical to the undivided
    bsn_add_self_gravity_source_f64 on every slab's cells."""
    import bsn
    from bsn import shard
    n, nz, d = 16, 32, (0.05, 0.07, 0.03)
    U = random_state(n, n, nz, seed=13, gamma=5 / 3)
    orc.fill_ghost_3d_outflow(U)
    Ud = dev(U)
    dU_ref = torch.zeros_like(Ud)
    bsn.add_self_gravity_source(dU_ref, Ud, n, n, nz, *d)
    ops = shard.DeviceOps()
    slabs = [shard.Slab.split(n, n, nz, r, world) for r in range(world)]
    P = [shard.SlabPoisson(s, *d, ops) for s in slabs]
    nzl = nz // world
    Us = []
    for s in slabs:
        V = bsn.state(n, n, nzl)
        shard._zmajor(V)[...] = shard._zmajor(Ud)[s.k0:s.k0 + nzl + 2 * NG]
        Us.append(V)
    sent = [P[r].forward(ops.active_rho(Us[r], n, n, nzl)) for r in range(world)]
    lines = [P[r].lines([sent[s][r] for s in range(world)]) for r in range(world)]
    phi = [P[r].inverse([lines[s][r] for s in range(world)]) for r in range(world)]
    for r, s in enumerate(slabs):
        lo = phi[r - 1].permute(2, 1, 0)[-1] if r > 0 else None
        hi = phi[r + 1].permute(2, 1, 0)[0] if r < world - 1 else None
        dUs = torch.zeros_like(Us[r])
        shard.sg_source(dUs, Us[r], phi[r], s, *d, ops, lo, hi)
        got = dUs[:, NG:NG + n, NG:NG + n, NG:NG + nzl]
        want = dU_ref[:, NG:NG + n, NG:NG + n, NG + s.k0:NG + s.k0 + nzl]
        assert torch.equal(got, want), (r, float((got - want).abs().max()))


def test_single_slab_self_gravity_step_matches_coupled_step(orc):
    """The sharded step with self-gravity on one rank (device operations,
    the distributed solve's phases) against the oracle's coupled_step! with
    no BHs: the FFTs differ by rounding only."""
    from bsn import shard
    n, nz, dx, g = 16, 16, 0.1, 5 / 3
    kw = dict(rho_floor=1e-8, P_floor=1e-8)
    U = random_state(n, n, nz, seed=19, gamma=g, jumps=False)
    orc.fill_ghost_3d_outflow(U)
    Ud = dev(U)
    slab = shard.Slab.split(n, n, nz, 0, 1)
    none = (orc.OrcBH * 1)()
    for _ in range(2):
        shard.euler3d_step(Ud, slab, dx, dx, dx, 1e-3, g, shard.DeviceOps(), self_gravity=True, **kw)
        orc.coupled_step(U, none, 0, 1e-3, 0.0, dx, 0.0, 0.0, 0.0, g, 1.0, kw["rho_floor"], kw["P_floor"],
                         True, True, 0.0, 0.0, evolve_orbit=False)
    got = host(Ud)
    a = (slice(NG, -NG),) * 3
    for q in range(5):
        assert np.abs(got[(q,) + a] - U[(q,) + a]).max() <= 1e-11 * np.abs(U[q]).max(), q
