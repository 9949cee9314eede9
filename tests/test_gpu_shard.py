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
