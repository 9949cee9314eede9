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


SLAB_SPECS = [dict(pos=(0.43, 0.37, 0.05), vel=(0.1, -0.2, 0.05), mass=1.0, eps=0.05, c_code=1e6, r_floor=0.3),
              dict(pos=(0.2, 0.61, -0.21), vel=(-0.1, 0.0, 0.2), mass=0.5, eps=0.02, c_code=1e6, r_floor=0.25)]


@pytest.mark.parametrize("world", [2, 4])
def test_slab_bh_sources_and_accretion_on_device(orc, world):
    """The slab forms of the BH sources on the device, the ranks' slabs taken
    one after another in one process: BH gravity and the sink sources with
    the global plane index are the undivided kernels' bit for bit, the
    accrete! terms of the slabs concatenated in rank order give the undivided
    accrete! (device and oracle) bit for bit, and the merged gas-force pairs
    agree with the undivided compensated sum to 1e-15."""
    import bsn
    from bsn import shard
    n, nz, d = 16, 32, (0.07, 0.08, 0.06)
    x0, y0, z0 = 0.0, -0.1, -0.96
    U = random_state(n, n, nz, seed=31)
    Ud = dev(U)
    mk = lambda: [bsn.BlackHole(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"])
                  for s in SLAB_SPECS]
    bhs = mk()
    dU_ref = torch.zeros_like(Ud)
    bsn.add_bh_gravity_source(dU_ref, Ud, n, n, nz, *d, bhs, x0, y0, z0)
    bsn.add_sink_sources(dU_ref, Ud, n, n, nz, *d, bhs, x0, y0, z0, f_sink=1.3, rho_sink_min=0.9)
    F_ref = [bsn.gas_force_on_bh(Ud, n, n, nz, *d, b, x0, y0, z0) for b in bhs]
    acc_ref = mk()
    for b in acc_ref:
        bsn.accrete(b, Ud, n, n, nz, *d, x0, y0, z0, 0.01, f_sink=1.3, rho_sink_min=0.9)
    nzl = nz // world
    pairs = [[] for _ in bhs]
    terms = [[] for _ in bhs]
    boxes = [bsn.sink_box(b, n, n, nz, *d, x0, y0, z0) for b in bhs]
    for r in range(world):
        k0 = r * nzl
        Us = bsn.state(n, n, nzl)
        shard._zmajor(Us)[...] = shard._zmajor(Ud)[k0:k0 + nzl + 2 * NG]
        dUs = torch.zeros_like(Us)
        bsn.add_bh_gravity_source_slab(dUs, Us, n, n, nzl, *d, bhs, x0, y0, z0, k0)
        bsn.add_sink_sources_slab(dUs, Us, n, n, nzl, *d, bhs, x0, y0, z0, k0, f_sink=1.3, rho_sink_min=0.9)
        got = dUs[:, NG:NG + n, NG:NG + n, NG:NG + nzl]
        want = dU_ref[:, NG:NG + n, NG:NG + n, NG + k0:NG + k0 + nzl]
        assert torch.equal(got, want), r
        for i, b in enumerate(bhs):
            pairs[i].append(bsn.gas_force_pairs_slab(Us, n, n, nzl, *d, b, x0, y0, z0, k0))
            terms[i].append(bsn.sink_terms_slab(Us, n, n, nzl, *d, x0, y0, z0, k0, b, 0.01, boxes[i], f_sink=1.3,
                                                rho_sink_min=0.9))
    assert sum(len(t) > 0 for t in terms[0]) >= 2   # the sphere straddles a slab boundary
    acc = mk()
    ob = [orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"]) for s in SLAB_SPECS]
    for i, b in enumerate(acc):
        bsn.accrete_from_terms(b, np.concatenate(terms[i]))
        orc.accrete(ob[i], U, *d, x0, y0, z0, 0.01, f_sink=1.3, rho_sink_min=0.9)
        assert b.mass > SLAB_SPECS[i]["mass"]
        for want in (acc_ref[i], ob[i]):
            assert b.mass == want.mass and list(b.vel) == list(want.vel)
        F = bsn.merge_force_pairs(np.array(pairs[i]))
        assert np.abs(F - F_ref[i]).max() <= 1e-15 * np.abs(F_ref[i]).max()
        s = SLAB_SPECS[i]   # the BH before accretion
        F_orc = orc.gas_force_on_bh(U, *d, orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"],
                                                       s["r_floor"]), x0, y0, z0)
        assert np.abs(F - F_orc).max() <= 1e-13 * np.abs(F_orc).max()


def test_single_slab_coupled_step_bitwise_to_oracle(orc):
    """shard.coupled_step on one rank with the device operations (the slab
    source forms, accrete! through its terms) against the oracle's
    coupled_step!, orbit frozen: bit for bit."""
    import bsn
    from bsn import shard
    from binary_ic import binary_setup
    U, dx, x0, specs = binary_setup(orc, n=32)
    Ud = dev(U)
    bg = [bsn.BlackHole(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"]) for s in specs]
    bo = orc.bh_array([orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"])
                       for s in specs])
    slab = shard.Slab.split(32, 32, 32, 0, 1)
    t = 0.0
    for _ in range(3):
        dt = orc.cfl_dt_3d(U, dx, dx, dx, 4 / 3, 0.4)
        shard.coupled_step(Ud, bg, slab, dt, t, dx, x0, x0, x0, 4 / 3, shard.DeviceOps(), rho_floor=1e-8,
                           P_floor=1e-10, rho_sink_min=2e-8, evolve_orbit=False)
        orc.coupled_step(U, bo, 2, dt, t, dx, x0, x0, x0, 4 / 3, 1.0, 1e-8, 1e-10, True, False, 0.0, 2e-8,
                         evolve_orbit=False)
        t += dt
    assert_bitwise(host(Ud), U, "coupled step on one slab")
    for i in range(2):
        assert bg[i].mass == bo[i].mass and list(bg[i].vel) == list(bo[i].vel)
        assert bg[i].mass > specs[i]["mass"]


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_fused_stages_equal_the_step(orc, precision):
    """bsn_euler3d_stage three times (ghosts filled by the caller, inputs and
    outputs alternating (a copy of U) -> A -> B -> U) is euler3d_step! of the same
    precision bit for bit; FP64 also equals the oracle."""
    import bsn
    n, dx, g = (14, 10, 12), 0.1, 1.4
    kw = dict(rho_floor=1e-6, P_floor=1e-5)
    U = random_state(*n, seed=51, vacuum=True)
    orc.fill_ghost_3d_outflow(U)
    dt = orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4)
    Ud, Us = dev(U), dev(U)
    (bsn.euler3d_step if precision == "f64" else bsn.euler3d_step_f32)(Ud, *n, dx, dx, dx, dt, g, **kw)
    C, A, B = Us.clone(), torch.zeros_like(Us), torch.zeros_like(Us)
    for s, (src, dst) in enumerate(((C, A), (A, B), (B, Us))):
        bsn.fill_ghost_3d_outflow(src, *n)
        bsn.euler3d_stage(dst, src, Us, *n, dx, dx, dx, dt, g, s + 1, precision=precision, **kw)
    assert torch.equal(Us, Ud)
    if precision == "f64":
        orc.euler3d_step(U, dx, dx, dx, dt, g, **kw)
        assert_bitwise(host(Us), U, "fused stages")


def test_single_slab_fp32_coupled_step_runs_the_fused_stage(orc):
    """The slab coupled step with FP32 stencils (one fused launch per stage,
    stiff faces in FP64 beside the sinks) stays within FP32 rounding of the
    oracle's FP64 coupled_step! over one step."""
    import bsn
    from bsn import shard
    from binary_ic import binary_setup
    U, dx, x0, specs = binary_setup(orc, n=32)
    Ud = dev(U)
    bg = [bsn.BlackHole(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"]) for s in specs]
    bo = orc.bh_array([orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"])
                       for s in specs])
    dt = orc.cfl_dt_3d(U, dx, dx, dx, 4 / 3, 0.4)
    shard.coupled_step(Ud, bg, shard.Slab.split(32, 32, 32, 0, 1), dt, 0.0, dx, x0, x0, x0, 4 / 3,
                       shard.DeviceOps(), rho_floor=1e-8, P_floor=1e-10, rho_sink_min=2e-8, evolve_orbit=False,
                       precision="f32")
    orc.coupled_step(U, bo, 2, dt, 0.0, dx, x0, x0, x0, 4 / 3, 1.0, 1e-8, 1e-10, True, False, 0.0, 2e-8,
                     evolve_orbit=False)
    G = host(Ud)
    a = (slice(NG, -NG),) * 3
    for q in (0, 4):
        err = np.abs(G[(q,) + a] - U[(q,) + a]).sum() / np.abs(U[(q,) + a]).sum()
        assert err < 1e-6, (q, err)
    assert abs(bg[0].mass - bo[0].mass) <= 1e-9 * bo[0].mass


def _blob(orc, n, nz, gamma):
    U = orc.state(n, n, nz)
    x = (np.arange(n) + 0.5) / n - 0.5
    z = (np.arange(nz) + 0.5) / nz - 0.5
    X, Y, Z = np.meshgrid(x, x, z, indexing="ij")
    rho = 1.0 + 4.0 * np.exp(-(X ** 2 + 2 * Y ** 2 + Z ** 2) / 0.02)
    vx, vy, vz = 0.1 * np.sin(2 * np.pi * Y), 0.1 * np.cos(2 * np.pi * Z), 0.05 * np.sin(2 * np.pi * X)
    a = (slice(NG, NG + n), slice(NG, NG + n), slice(NG, NG + nz))
    U[(0,) + a], U[(1,) + a], U[(2,) + a], U[(3,) + a] = rho, rho * vx, rho * vy, rho * vz
    U[(4,) + a] = 1.0 / (gamma - 1.0) + 0.5 * rho * (vx ** 2 + vy ** 2 + vz ** 2)
    orc.fill_ghost_3d_outflow(U)
    return U


@pytest.mark.parametrize("self_gravity", [False, True])
def test_single_slab_fmr_step_bitwise_to_the_device_step(orc, self_gravity):
    """The slab FMR step (bsn/shard_fmr.py) on one rank through the library's
    operators -- coarse stages with the register faces, the owner's window,
    fine subcycles, restriction and Berger-Colella correction -- equals the
    fused bsn_fmr3d_step_f64 bit for bit (64^3 coarse, 64^3 fine patch)."""
    import bsn
    from bsn import shard, shard_fmr
    n, dxc, g, r = 64, 1.0 / 32.0, 5.0 / 3.0, 2
    box = (17, 48, 17, 48, 17, 48)
    kw = dict(rho_floor=1e-6, P_floor=1e-5)
    U0 = _blob(orc, n, n, g)
    Gd = bsn.FMRGrid3D(dev(U0), n, n, n, dxc, *box, r, g, **kw)
    slab = shard.Slab.split(n, n, n, 0, 1)
    S = shard_fmr.SlabFMR(dev(U0), slab, dxc, *box, r, g, shard.DeviceOps(), Uf=Gd.Uf.clone(), **kw)
    for _ in range(3):
        dt = bsn.cfl_dt_fmr3d(Gd, 0.4)
        assert S.cfl_dt(0.4) == dt
        S.step(dt, self_gravity=self_gravity, G_grav=0.5)
        bsn.fmr3d_step(Gd, dt, self_gravity=self_gravity, G_grav=0.5)
    a = (slice(None),) + (slice(NG, -NG),) * 3
    assert torch.equal(S.Uc[a], Gd.Uc[a])
    assert torch.equal(S.G.Uf[a], Gd.Uf[a])
