"""FP64 parity with the oracle at the workloads' own sizes.

The other parity tests run at sizes chosen for coverage of branches; these
run the FP64 device path and the oracle side by side on the full-size inputs
of the Sedov, polytrope and binary-BH workloads, one to three steps each
(what the oracle's CPU threads finish in seconds):

* Sedov blast 128^3 on [-1,1]^3 (gamma 5/3, E = 1 in r < 3.5 dx, floors 1e-6):
  three CFL-limited euler3d_step! steps, bit-identical (dt included);
* n = 1 polytrope (M = 1, R = 0.5, gamma 2) in a 1e-8 atmosphere, base 128^3
  on [-2,2]^3 with a 128^3 patch on [-1,1]^3 (ratio 2), with and without the
  rigid rotation Omega = 0.2 of breakup: one fmr3d_step! with self-gravity
  through the host-driven entry and through the graph-captured device loop,
  within 1e-12 relative L-inf of each conserved field (the FFT sums round
  differently from the oracle's; every other operation is bit-identical;
  momenta relative to the largest momentum the state's energy allows);
* binary BH supernova on three nested 128^3 levels ([-8,8]^3, [-4,4]^3,
  [-2,2]^3): n = 3 polytrope M = 10, R = 1, thermal bomb E = 1 in r < 0.1,
  two m = 5 sinks at (+-1.5, 0, 0) on their circular orbit, sink radius 4
  finest cells: one coupled step with the orbit frozen and no self-gravity
  bit-identical; with the live orbit and self-gravity within 1e-12 relative
  L-inf per field on every level.
"""
import math
import os

import numpy as np
import pytest

from binary_ic import binary_nested_setup
from gpu_util import NG, assert_bitwise, dev, host

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def bsn():
    import bsn as b
    return b


@pytest.fixture(scope="module", autouse=True)
def _oracle_threads(orc):
    orc.set_threads(os.cpu_count() or 1)


def _linf_per_field(got, want):
    """max |got - want| over each conserved field, relative to the field's
    scale: max |rho| and max |E| for density and energy; for the momenta
    max sqrt(2 rho E), the largest momentum the state's energy allows
    (|m| <= sqrt(2 rho E) since E >= m^2 / (2 rho)).  A star in hydrostatic
    equilibrium has momenta at the rounding level of the pressure-gravity
    cancellation (1e-16 of rho g dt), so their own maximum is no scale."""
    mscale = float(np.sqrt(2.0 * np.abs(want[0] * want[4])).max())
    scale = [np.abs(want[0]).max(), mscale, mscale, mscale, np.abs(want[4]).max()]
    return [float(np.abs(got[q] - want[q]).max() / max(scale[q], 1e-300)) for q in range(5)]


def test_sedov128_fp64_steps_bitwise(orc, bsn):
    n, g, L = 128, 5.0 / 3.0, 1.0
    dx = 2 * L / n
    kw = dict(rho_floor=1e-6, P_floor=1e-6)
    U = orc.state(n, n, n)
    orc.sedov_ic_3d(U, dx, dx, dx, g, E_blast=1.0, r_inject=3.5 * dx, rho_bg=1.0, P_floor=1e-5,
                    x_offset=-L, y_offset=-L, z_offset=-L)
    Ud = dev(U)
    for step in range(3):
        dt = orc.cfl_dt_3d(U, dx, dx, dx, g, 0.4)
        assert bsn.cfl_dt_3d(Ud, n, n, n, dx, dx, dx, g, 0.4) == dt, step
        orc.euler3d_step(U, dx, dx, dx, dt, g, **kw)
        bsn.euler3d_step(Ud, n, n, n, dx, dx, dx, dt, g, **kw)
    assert_bitwise(host(Ud), U, "Sedov 128^3 after three steps")


def _polytrope_fmr(orc, bsn, omega_frac):
    from bsn import ics
    nc, ratio, g = 128, 2, 2.0
    dxc = 4.0 / nc
    lo, hi = 33, 96
    kw = dict(rho_floor=1e-8, P_floor=1e-10)
    Uc = orc.state(nc, nc, nc)
    orc.polytrope_ic_3d(Uc, dxc, dxc, dxc, g, 1.0, 0.5, x0=-2.0, y0=-2.0, z0=-2.0, **kw)
    if omega_frac:
        ics.apply_stellar_rotation(Uc, nc, nc, nc, dxc, g, omega_frac * math.sqrt(1.0 / 0.5 ** 3),
                                   rho_thresh=2e-8, x0=-2.0, y0=-2.0)
    orc.fill_ghost_3d_outflow(Uc)
    Go = orc.FMRGrid(Uc.copy(order="F"), dxc, lo, hi, lo, hi, lo, hi, ratio, g, **kw)
    grids = [bsn.FMRGrid3D(dev(Uc), nc, nc, nc, dxc, lo, hi, lo, hi, lo, hi, ratio, g, **kw) for _ in range(2)]
    return Go, grids


@pytest.mark.parametrize("omega_frac", [0.0, 0.2])
def test_polytrope_fmr128_selfgravity_step(orc, bsn, omega_frac):
    Go, (Gd, Gl) = _polytrope_fmr(orc, bsn, omega_frac)
    assert_bitwise(host(Gd.Uf), Go.Uf, "prolonged patch")
    dt = Go.cfl_dt(0.4)
    assert bsn.cfl_dt_fmr3d(Gd, 0.4) == dt
    Go.step(dt, self_gravity=True)
    bsn.fmr3d_step(Gd, dt, self_gravity=True)
    t, k = bsn.fmr3d_run_steps(Gl, 0.4, n_steps=1, precision="f64", self_gravity=True)
    assert k == 1 and t == dt
    for G in (Gd, Gl):
        for name, A, B in (("coarse", host(G.Uc), Go.Uc), ("fine", host(G.Uf), Go.Uf)):
            err = _linf_per_field(A, B)
            assert max(err) <= 1e-12, (name, err)


def _nested(orc, bsn):
    H, boxes, dx0, x0, specs = binary_nested_setup(orc, n=128, L=8.0, sep=3.0, r_bomb=0.1, sink_cells=4)
    n = 128
    Hd = bsn.FMRHierarchy3D(dev(H.levels[0]), n, n, n, dx0, boxes, 4 / 3, rho_floor=1e-8, P_floor=1e-10,
                            init=False)
    for Ud, Uo in zip(Hd.levels, H.levels):
        Ud.copy_(dev(Uo))
    bo = orc.bh_array([orc.make_bh(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"])
                       for s in specs])
    bg = [bsn.BlackHole(s["pos"], s["vel"], s["mass"], s["eps"], s["c_code"], s["r_floor"]) for s in specs]
    return H, Hd, bo, bg, x0


@pytest.mark.parametrize("live", [False, True])
def test_binary_nested128_coupled_step(orc, bsn, live):
    H, Hd, bo, bg, x0 = _nested(orc, bsn)
    dt = H.cfl_dt(0.4)
    H.coupled_step(bo, 2, dt, 0.0, x0, x0, x0, 1.0, True, live, 0.0, 0.0, evolve_orbit=live)
    t, k = bsn.coupled_nested_run_steps(Hd, bg, x0, x0, x0, 0.4, n_steps=1, f_sink=1.0, torque_free=True,
                                        self_gravity=live, rho_sink_min=0.0, evolve_orbit=live)
    assert k == 1 and t == dt
    for lev, (Ud, Uo) in enumerate(zip(Hd.levels, H.levels)):
        if live:
            err = _linf_per_field(host(Ud), Uo)
            assert max(err) <= 1e-12, (lev, err)
        else:
            assert_bitwise(host(Ud), Uo, f"level {lev}")
    for i in range(2):
        if live:
            assert abs(bg[i].mass - bo[i].mass) <= 1e-14 * bo[i].mass
            assert max(abs(a - b) for a, b in zip(bg[i].pos, bo[i].pos)) <= 1e-14
        else:
            assert bg[i].mass == bo[i].mass and list(bg[i].vel) == list(bo[i].vel)
