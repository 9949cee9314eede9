"""The product's initial-condition generators (bsn.ics) against the oracle's
restatement of the reference IC functions: bit-identical states."""
import numpy as np
import pytest

import importlib.util
import os

_spec = importlib.util.spec_from_file_location(
    "bsn_ics", os.path.join(os.path.dirname(__file__), "..", "binary-supernova_b200", "bsn", "ics.py"))
ics = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(ics)


def _eq(a, b):
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("n,off", [(24, -1.0), (17, -0.5)])
def test_sedov(orc, n, off):
    dx = 2.0 / n
    A = orc.state(n, n + 1, n + 2)
    orc.sedov_ic_3d(A, dx, dx, dx, 5 / 3, E_blast=1.0, r_inject=3.5 * dx, rho_bg=1.0, P_floor=1e-5,
                    x_offset=off, y_offset=off, z_offset=off)
    B = orc.state(n, n + 1, n + 2)
    ics.sedov_ic_3d(B, n, n + 1, n + 2, dx, dx, dx, 5 / 3, E_blast=1.0, r_inject=3.5 * dx, rho_bg=1.0,
                    P_floor=1e-5, x_offset=off, y_offset=off, z_offset=off)
    _eq(A, B)


@pytest.mark.parametrize("d", ["x", "y", "z"])
def test_sod(orc, d):
    A, dims, dxs = orc.sod_ic_3d(d, n_normal=32, n_trans=4)
    B = orc.state(*dims)
    assert ics.sod_ic_3d(B, *dims, direction=d) == dxs
    _eq(A, B)


@pytest.mark.parametrize("gamma,M,R", [(2.0, 1.0, 0.5), (4 / 3, 10.0, 1.0)])
def test_polytrope_and_bomb(orc, gamma, M, R):
    n, L = 20, 2.0
    dx = 2 * L / n
    A = orc.state(n, n, n)
    outA = orc.polytrope_ic_3d(A, dx, dx, dx, gamma, M, R, x0=-L, y0=-L, z0=-L, rho_floor=1e-8, P_floor=1e-10)
    B = orc.state(n, n, n)
    outB = ics.polytrope_ic_3d(B, n, n, n, dx, dx, dx, gamma, M_star=M, R_star=R, x0=-L, y0=-L, z0=-L,
                               rho_floor=1e-8, P_floor=1e-10)
    assert tuple(outA) == tuple(outB)
    _eq(A, B)
    mA = orc.thermal_bomb(A, dx, dx, dx, 1.0, 0.5, x0=-L, y0=-L, z0=-L)
    mB = ics.thermal_bomb(B, n, n, n, dx, dx, dx, E_SN=1.0, r_bomb=0.5, x0=-L, y0=-L, z0=-L)
    assert mA == mB
    _eq(A, B)


def test_bomb_without_gas_raises():
    B = np.zeros((5, 14, 14, 14), order="F")
    with pytest.raises(ValueError):
        ics.thermal_bomb(B, 8, 8, 8, 0.1, 0.1, 0.1, E_SN=1.0, r_bomb=0.2)


def test_stellar_rotation_overlay(orc):
    """apply_stellar_rotation! (scripts/run_sn50_fiducial.jl:421-446) as the
    reference's cell loop, written out here in plain Python at a small size:
    the vectorised overlay must produce the same bits."""
    n, g, dx, x0 = 12, 2.0, 4.0 / 12, -2.0
    A = orc.state(n, n + 2, n + 1)
    orc.polytrope_ic_3d(A, dx, dx, dx, g, 1.0, 1.2, x0=x0, y0=x0, z0=x0, rho_floor=1e-8, P_floor=1e-10)
    B = A.copy(order="F")
    Om, vsy, xs, ys, thr = 0.5657, 0.1, 0.05, -0.02, 2e-8
    NG = 3
    for k in range(NG, NG + n + 1):
        for j in range(NG, NG + n + 2):
            for i in range(NG, NG + n):
                rho = A[0, i, j, k]
                if rho <= thr:
                    continue
                xc = x0 + (i + 1 - NG - 0.5) * dx - xs
                yc = x0 + (j + 1 - NG - 0.5) * dx - ys
                vx, vy, vz = -Om * yc, vsy + Om * xc, 0.0
                P = A[4, i, j, k] * (g - 1.0)
                A[1, i, j, k], A[2, i, j, k], A[3, i, j, k] = rho * vx, rho * vy, rho * vz
                A[4, i, j, k] = P / (g - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    ics.apply_stellar_rotation(B, n, n + 2, n + 1, dx, g, Om, v_star_y=vsy, x_star=xs, y_star=ys, rho_thresh=thr,
                               x0=x0, y0=x0)
    assert (A[0] > thr).sum() > 100
    _eq(A, B)
