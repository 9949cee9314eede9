"""Two-level FMR with the coarse level in z-slabs (bsn/shard_fmr.py) on CPU:
two or four gloo ranks step their coarse slabs with the oracle's operators and
the owner rank steps the refined patch from its window of the coarse grid.
Without self-gravity every slab and the fine level must equal the oracle's
undivided fmr3d_step! (src/fmr3d.jl:451-604) bit for bit, with the same dts;
with self-gravity (the distributed solve's phases through torch.fft) the
slabs must equal the same code run undivided bit for bit, and the oracle's
own step within the two FFTs' rounding."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NG = 3
N, NZG, DXC, GAMMA, RATIO = 16, 32, 1.0 / 16.0, 1.4, 2
BOX = (5, 12, 5, 12, 10, 21)
KW = dict(rho_floor=1e-6, P_floor=1e-5)


def _smooth(orc):
    """A smooth self-gravitating blob (the random state's reconstructions are
    too ill-conditioned to compare two FFTs' rounding through a step)."""
    U = orc.state(N, N, NZG)
    x = (np.arange(N) + 0.5) / N - 0.5
    z = (np.arange(NZG) + 0.5) / NZG - 0.5
    X, Y, Z = np.meshgrid(x, x, 2 * z, indexing="ij")
    rho = 1.0 + 4.0 * np.exp(-(X ** 2 + 2 * Y ** 2 + Z ** 2) / 0.05)
    vx, vy, vz = 0.1 * np.sin(2 * np.pi * Y), 0.1 * np.cos(2 * np.pi * Z), 0.05 * np.sin(2 * np.pi * X)
    a = (slice(NG, NG + N), slice(NG, NG + N), slice(NG, NG + NZG))
    U[(0,) + a], U[(1,) + a], U[(2,) + a], U[(3,) + a] = rho, rho * vx, rho * vy, rho * vz
    U[(4,) + a] = 1.0 / (GAMMA - 1.0) + 0.5 * rho * (vx ** 2 + vy ** 2 + vz ** 2)
    orc.fill_ghost_3d_outflow(U)
    return U


def _setup(orc, smooth=False, box=BOX):
    from test_shard import _initial
    U = _smooth(orc) if smooth else _initial(orc, N, NZG, 11, "outflow")
    G = orc.FMRGrid(U.copy(order="F"), DXC, *box, RATIO, GAMMA, **KW)
    return U, G


def _slab_grid(orc, shard, shard_fmr, U0, Uf0, rank, world, ops, owner, box=BOX):
    slab = shard.Slab.split(N, N, NZG, rank, world)
    Us = orc.state(N, N, slab.nz)
    Us[...] = U0[:, :, :, slab.k0:slab.k0 + slab.nz + 2 * NG]
    S = shard_fmr.SlabFMR(Us, slab, DXC, *box, RATIO, GAMMA, ops, owner=owner, Uf=Uf0, **KW)
    return slab, S


def _fmr_worker(rank, world, port, q, self_gravity, owner, box=BOX):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        import torch.distributed as dist
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        sys.path.insert(0, os.path.join(ROOT, "binary-supernova_b200"))
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle as orc
        from bsn import shard, shard_fmr
        from test_shard import OracleOps, SGOps
        dist.init_process_group("gloo", rank=rank, world_size=world)
        U0, G = _setup(orc, smooth=self_gravity, box=box)
        Uf0 = G.Uf.copy(order="F")
        ops = SGOps(orc) if self_gravity else OracleOps(orc, DXC)
        slab, S = _slab_grid(orc, shard, shard_fmr, U0, Uf0, rank, world, ops, owner, box)
        # the undivided reference: the oracle's step, and (self-gravity) the
        # same slab code on one rank
        W = None
        if self_gravity:
            _, W = _slab_grid(orc, shard, shard_fmr, U0, Uf0, 0, 1, ops, 0)
        info, ok = [], True
        for _ in range(2):
            dt = G.cfl_dt(0.4)
            dts = S.cfl_dt(0.4)
            # every rank takes the undivided grid's dt (with self-gravity the
            # undivided run of the same code's: the oracle's differs by its FFT's rounding)
            ok &= dts == (W.cfl_dt(0.4) if W is not None else dt)
            S.step(dt, self_gravity=self_gravity)
            G.step(dt, self_gravity=self_gravity)
            if W is not None:
                W.step(dt, self_gravity=True)
        k0, nz = slab.k0, slab.nz
        act = (slice(None), slice(NG, NG + N), slice(NG, NG + N))
        mine = S.Uc[act + (slice(NG, NG + nz),)]
        ref_c = (W.Uc if W is not None else G.Uc)[act + (slice(NG + k0, NG + k0 + nz),)]
        ok &= bool(np.array_equal(mine, ref_c))
        info.append(float(np.abs(mine - ref_c).max()))
        if rank == owner:
            fa = (slice(None),) + (slice(NG, -NG),) * 3
            ref_f = (W.G.Uf if W is not None else G.Uf)[fa]
            ok &= bool(np.array_equal(S.G.Uf[fa], ref_f))
            info.append(float(np.abs(S.G.Uf[fa] - ref_f).max()))
        if self_gravity:   # the oracle's step (its own FFT) within rounding
            oc = G.Uc[act + (slice(NG + k0, NG + k0 + nz),)]
            err = float(np.abs(mine - oc).max() / np.abs(oc).max())
            ok &= err < 1e-12
            info.append(err)
        q.put((rank, ok, info))
        dist.destroy_process_group()
    except Exception as e:   # report to the parent instead of hanging it
        import traceback
        q.put((rank, False, traceback.format_exc()))


@pytest.mark.parametrize("world,owner", [(2, 0), (2, 1), (4, 2)])
def test_slab_fmr_step_matches_the_undivided_step(world, owner):
    from test_shard import _spawn
    for rank, ok, info in _spawn(_fmr_worker, world, (False, owner)):
        assert ok, (rank, info)


def test_slab_fmr_owner_outside_the_window():
    """The owner holds none of the window's planes (rank 0 of 4 owns planes
    1-8; the window of a box on planes 18-23 is 10-31): it still gathers,
    steps the patch and sends the planes back."""
    from test_shard import _spawn
    for rank, ok, info in _spawn(_fmr_worker, 4, (False, 0, (4, 11, 6, 13, 18, 23))):
        assert ok, (rank, info)


@pytest.mark.parametrize("world", [2, 4])
def test_slab_fmr_step_with_self_gravity(world):
    from test_shard import _spawn
    for rank, ok, info in _spawn(_fmr_worker, world, (True, 0)):
        assert ok, (rank, info)


def test_slab_fmr_checks(orc):
    sys.path.insert(0, os.path.join(ROOT, "binary-supernova_b200"))
    from bsn import shard, shard_fmr
    from test_shard import OracleOps
    U0, G = _setup(orc)
    ops = OracleOps(orc, DXC)
    slab = shard.Slab.split(N, N, NZG, 0, 1)
    with pytest.raises(ValueError):   # the window would reach past the z boundary
        shard_fmr.SlabFMR(U0, slab, DXC, 5, 12, 5, 12, 4, 21, RATIO, GAMMA, ops)
    with pytest.raises(ValueError):
        shard_fmr.SlabFMR(U0, slab, DXC, 5, 17, 5, 12, 10, 21, RATIO, GAMMA, ops)
    per = shard.Slab.split(N, N, NZG, 0, 1, "periodic")
    with pytest.raises(ValueError):
        shard_fmr.SlabFMR(U0, per, DXC, *BOX, RATIO, GAMMA, ops)
