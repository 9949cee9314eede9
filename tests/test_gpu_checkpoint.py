"""Restart from a checkpoint in the reference's HDF5 layout is bit-exact on
the device: the coupled driver loop (sinks, live orbit, self-gravity) run for
six steps equals three steps, an asynchronous checkpoint taken while three
more steps run on the same state, and a restart from the file for the last
three (src/checkpoint.jl: "so the restart is bit-for-bit faithful")."""
import numpy as np
import pytest

from gpu_util import dev, host

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _bhs(bsn, specs):
    return [bsn.BlackHole(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"]) for s in specs]


def test_restart_from_async_checkpoint_is_bitwise(orc, tmp_path):
    import bsn
    from binary_ic import binary_setup
    n = 32
    U, dx, x0, specs = binary_setup(orc, n=n)
    kw = dict(f_sink=1.0, rho_floor=1e-8, P_floor=1e-10, torque_free=True, self_gravity=True, rho_sink_min=2e-8,
              evolve_orbit=True)
    geo = (n, n, n, dx, x0, x0, x0, 4 / 3, 0.4)
    Ua, ba = dev(U), _bhs(bsn, specs)
    ta, na = bsn.coupled_run_steps(Ua, ba, *geo, n_steps=6, **kw)
    Ub, bb = dev(U), _bhs(bsn, specs)
    tb, _ = bsn.coupled_run_steps(Ub, bb, *geo, n_steps=3, **kw)
    p = tmp_path / "restart.h5"
    bsn.save_checkpoint_uniform(p, Ub, bb, t=tb, step=3, dt_last=0.0, t_snap=0.0, t_bh2_sink_on=0.0, nx=n, ny=n,
                                nz=n, dx=dx, dy=dx, dz=dx, gamma=4 / 3, x0=x0, y0=x0, z0=x0, rho_floor=1e-8,
                                P_floor=1e-10, asynchronous=True)
    tb2, _ = bsn.coupled_run_steps(Ub, bb, *geo, n_steps=3, t=tb, **kw)   # runs on while the file is written
    bsn.checkpoint_wait()
    assert tb2 == ta and torch.equal(Ub, Ua)
    Uc, bc, grid, meta = bsn.load_checkpoint_uniform(p)
    assert meta["t"] == tb and meta["step"] == 3 and grid["nx"] == n and grid["dx"] == dx
    tc, nc = bsn.coupled_run_steps(Uc, bc, *geo, n_steps=3, t=meta["t"], **kw)
    assert (tc, nc) == (ta, 3)
    assert torch.equal(Uc, Ua)
    for a, b in zip(bc, ba):
        assert list(a.pos) == list(b.pos) and list(a.vel) == list(b.vel) and a.mass == b.mass


def test_fmr_checkpoint_round_trip_on_device(orc, tmp_path):
    import bsn
    from gpu_util import random_state
    U = random_state(16, 16, 16, seed=41)
    orc.fill_ghost_3d_outflow(U)
    G = bsn.FMRGrid3D(dev(U), 16, 16, 16, 0.125, 5, 12, 4, 11, 6, 13, 2, 5 / 3, rho_floor=1e-8, P_floor=1e-10)
    G.Uf.add_(torch.rand_like(G.Uf) * 1e-3)   # a fine level that is not the prolongation
    bhs = [bsn.BlackHole((0.1, 0.2, 0.3), (0.0, 1.0, 0.0), 2.0, 0.05, 1e6, 0.2)]
    p = tmp_path / "fmr.h5"
    bsn.save_checkpoint(p, G, bhs, t=0.25, step=17, dt_last=1e-3)
    H, bh2, meta = bsn.load_checkpoint(p)
    assert meta == dict(t=0.25, step=17, dt_last=1e-3, format_version=1)
    assert torch.equal(H.Uc, G.Uc) and torch.equal(H.Uf, G.Uf)
    for f in ("ncx", "ncy", "ncz", "nfx", "nfy", "nfz", "ratio", "ci_lo", "ci_hi", "cj_lo", "cj_hi", "ck_lo",
              "ck_hi", "bc", "dxc", "dyc", "dzc", "dxf", "dyf", "dzf", "gamma", "rho_floor", "P_floor"):
        assert getattr(H.s, f) == getattr(G.s, f), f
    assert list(bh2[0].pos) == [0.1, 0.2, 0.3] and bh2[0].mass == 2.0
    # a device snapshot of the coarse level reads back as its active cells
    q = tmp_path / "snap.h5"
    bsn.write_snapshot(q, G.Uc, 16, 16, 16, 0.125, 0.125, 0.125, 0.25, 5 / 3)
    A = bsn.read_snapshot(q)[0]
    assert np.array_equal(A, host(G.Uc)[:, 3:-3, 3:-3, 3:-3])
