"""Initial conditions of the workloads, written into a state in the
reference layout U[q, i, j, k] (ghost width NG = 3, active cells
NG..NG+n-1), either a device tensor from bsn.state() or a host numpy array of
shape (5, nx+6, ny+6, nz+6) in column-major (Fortran) order.

The fields are computed on the host in FP64 with the reference's operation
order, so the states are bit-identical to the reference's (the sums over
cells -- the Sedov injection volume, the thermal-bomb mass -- accumulate
sequentially in the reference's loop order i fastest, then j, then k):

* sedov_ic_3d      src/euler3d.jl:275-316 (sedov_ic_3d!)
* sod_ic_3d        test/test_sod3d.jl:86-104 (_run_sod_3d initial state)
* lane_emden       src/stellar_ic.jl:34-63
* polytrope_ic_3d  src/stellar_ic.jl:87-178 (polytrope_ic_3d!)
* thermal_bomb     src/stellar_ic.jl:210-253 (thermal_bomb!)
* apply_stellar_rotation  scripts/run_sn50_fiducial.jl:421-446
                   (apply_stellar_rotation!, the rigid-rotation overlay)
"""
from __future__ import annotations

import math

import numpy as np

NG = 3


def _host_like(U, nx, ny, nz):
    shape = (5, nx + 2 * NG, ny + 2 * NG, nz + 2 * NG)
    if tuple(U.shape) != shape:
        raise ValueError(f"state has shape {tuple(U.shape)}, expected {shape}")
    if isinstance(U, np.ndarray):
        if not U.flags.f_contiguous or U.dtype != np.float64:
            raise ValueError("host state must be a column-major float64 array")
        return U
    return np.zeros(shape, dtype=np.float64, order="F")


def _store(U, H):
    if H is not U:
        import torch
        U.copy_(torch.from_numpy(H))


def _read(U, nx, ny, nz):
    if isinstance(U, np.ndarray):
        return U
    H = np.zeros((5, nx + 2 * NG, ny + 2 * NG, nz + 2 * NG), dtype=np.float64, order="F")
    import torch
    torch.from_numpy(H).copy_(U.cpu())
    return H


def _r2(xc, yc, zc):
    """xc^2 + yc^2 + zc^2 over the active block, (x*x + y*y) + z*z."""
    return (xc[:, None, None] * xc[:, None, None] + yc[None, :, None] * yc[None, :, None]) + \
        zc[None, None, :] * zc[None, None, :]


def _seq_sum(v: np.ndarray) -> float:
    """Left-to-right sum (the reference's loop accumulation)."""
    if v.size == 0:
        return 0.0
    return float(np.add.accumulate(v.ravel(order="F"))[-1])


def sedov_ic_3d(U, nx, ny, nz, dx, dy, dz, gamma, *, E_blast=1.0, r_inject=None, rho_bg=1.0, P_floor=1e-5,
                x_offset=0.0, y_offset=0.0, z_offset=0.0):
    """sedov_ic_3d! (src/euler3d.jl:275-316): background rho_bg, P_floor;
    E_blast (gamma-1)/V_inj added to the energy of the cells with r <= r_inject."""
    H = _host_like(U, nx, ny, nz)
    H[...] = 0.0
    r_inj = 2.5 * min(dx, dy, dz) if r_inject is None else float(r_inject)
    a = (slice(NG, NG + nx), slice(NG, NG + ny), slice(NG, NG + nz))
    E_bg = P_floor / (gamma - 1)
    xc = (np.arange(1, nx + 1, dtype=np.float64) - 0.5) * dx + x_offset
    yc = (np.arange(1, ny + 1, dtype=np.float64) - 0.5) * dy + y_offset
    zc = (np.arange(1, nz + 1, dtype=np.float64) - 0.5) * dz + z_offset
    inside = np.sqrt(_r2(xc, yc, zc)) <= r_inj
    cnt = int(inside.sum())
    V_inj = _seq_sum(np.full(cnt, dx * dy * dz))
    dE = E_blast * (gamma - 1) / V_inj if V_inj > 0.0 else 0.0
    H[(0,) + a] = rho_bg
    H[(4,) + a] = np.where(inside, E_bg + dE, E_bg)
    _store(U, H)


def sod_ic_3d(U, nx, ny, nz, direction="x", gamma=1.4):
    """Sod initial state of test/test_sod3d.jl:86-104 on [0,1]^3 split at 0.5
    along `direction`: (rho, v, p) = (1, 0, 1) left, (0.125, 0, 0.1) right.
    Returns (dx, dy, dz)."""
    H = _host_like(U, nx, ny, nz)
    H[...] = 0.0
    dx, dy, dz = 1.0 / nx, 1.0 / ny, 1.0 / nz
    ax = "xyz".index(direction)
    n, d = (nx, ny, nz)[ax], (dx, dy, dz)[ax]
    coord = (np.arange(1, n + 1, dtype=np.float64) - 0.5) * d - 0.5
    left = coord < 0.0
    rho = np.where(left, 1.0, 0.125)
    E = np.where(left, 1.0, 0.1) / (gamma - 1) + 0.5 * rho * 0.0 ** 2
    shape = [1, 1, 1]
    shape[ax] = n
    a = (slice(NG, NG + nx), slice(NG, NG + ny), slice(NG, NG + nz))
    H[(0,) + a] = np.broadcast_to(rho.reshape(shape), (nx, ny, nz))
    H[(4,) + a] = np.broadcast_to(E.reshape(shape), (nx, ny, nz))
    _store(U, H)
    return dx, dy, dz


def lane_emden(n: float, dxi: float = 1e-3):
    """RK4 solution of the Lane-Emden equation of index n from a Taylor seed
    at xi = dxi until theta <= 0 (src/stellar_ic.jl:34-63).  Returns
    (xis, thetas, dthetas) as float64 arrays."""
    nf = float(n)
    xi0 = dxi
    th0 = 1.0 - xi0 * xi0 / 6.0 + nf * ((xi0 * xi0) * (xi0 * xi0)) / 120.0
    dth0 = -xi0 / 3.0 + nf * (xi0 * xi0 * xi0) / 30.0

    def f(xi, th, dth):
        return -math.pow(max(th, 0.0), nf) - 2.0 * dth / xi

    xis, ths, dths = [xi0], [th0], [dth0]
    xi, th, dth = xi0, th0, dth0
    while th > 0.0:
        k1t = dxi * dth
        k1d = dxi * f(xi, th, dth)
        k2t = dxi * (dth + k1d / 2)
        k2d = dxi * f(xi + dxi / 2, th + k1t / 2, dth + k1d / 2)
        k3t = dxi * (dth + k2d / 2)
        k3d = dxi * f(xi + dxi / 2, th + k2t / 2, dth + k2d / 2)
        k4t = dxi * (dth + k3d)
        k4d = dxi * f(xi + dxi, th + k3t, dth + k3d)
        th += (k1t + 2 * k2t + 2 * k3t + k4t) / 6
        dth += (k1d + 2 * k2d + 2 * k3d + k4d) / 6
        xi += dxi
        xis.append(xi)
        ths.append(th)
        dths.append(dth)
    return np.array(xis), np.array(ths), np.array(dths)


def polytrope_ic_3d(U, nx, ny, nz, dx, dy, dz, gamma, *, M_star, R_star, M_core=0.0, x0=0.0, y0=0.0, z0=0.0,
                    x_center=0.0, y_center=0.0, z_center=0.0, rho_floor=1e-10, P_floor=1e-8):
    """polytrope_ic_3d! (src/stellar_ic.jl:87-178): Lane-Emden polytrope of
    index 1/(gamma-1), mass M_star, radius R_star (G = 1), zero velocity, floor
    values outside R_star and inside the carved core of mass M_core.
    Returns (rho_c, r_scale, K, r_core)."""
    H = _host_like(U, nx, ny, nz)
    n = 1.0 / (gamma - 1.0)
    xis, ths, dths = lane_emden(n)
    xi1, dth1 = xis[-1], dths[-1]
    omega_n = -(xi1 * xi1) * dth1
    r_scale = R_star / xi1
    rho_c = M_star / (4.0 * math.pi * (r_scale * r_scale * r_scale) * omega_n)
    K = 4.0 * math.pi * (r_scale * r_scale) * math.pow(rho_c, 1.0 - 1.0 / n) / (n + 1.0)
    dxs = xis[1] - xis[0]
    N = len(xis)

    r_core = 0.0
    if M_core > 0.0:
        if not M_core < M_star:
            raise ValueError(f"polytrope_ic_3d: M_core ({M_core}) >= M_star ({M_star})")
        target = float(M_core) / float(M_star)
        xi_core = xi1
        for i in range(N):
            frac = -(xis[i] * xis[i]) * dths[i] / omega_n
            if frac >= target:
                if i > 0:
                    f0 = -(xis[i - 1] * xis[i - 1]) * dths[i - 1] / omega_n
                    al = (target - f0) / (frac - f0)
                    xi_core = xis[i - 1] + al * (xis[i] - xis[i - 1])
                else:
                    xi_core = xis[i]
                break
        r_core = xi_core * r_scale
    r_core2 = r_core * r_core

    xc = x0 + (np.arange(1, nx + 1, dtype=np.float64) - 0.5) * dx - x_center
    yc = y0 + (np.arange(1, ny + 1, dtype=np.float64) - 0.5) * dy - y_center
    zc = z0 + (np.arange(1, nz + 1, dtype=np.float64) - 0.5) * dz - z_center
    r2 = _r2(xc, yc, zc)
    xq = np.sqrt(r2) / r_scale
    i_f = xq / dxs
    i = np.clip(np.floor(i_f), 1, N - 1).astype(np.int64)
    al = i_f - i
    th = (1.0 - al) * ths[i - 1] + al * ths[i]
    th = np.where(xq <= 0.0, 1.0, np.where(xq >= xi1, 0.0, th))
    star = (th > 0.0) & (r2 >= r_core2)
    rho = np.full(r2.shape, float(rho_floor))
    P = np.full(r2.shape, float(P_floor))
    ts = th[star]
    # math.pow per star cell: the C library's pow, as the reference's ^
    rs = np.array([rho_c * math.pow(t, n) for t in ts.tolist()], dtype=np.float64)
    rho[star] = rs
    P[star] = np.array([K * math.pow(r, 1.0 + 1.0 / n) for r in rs.tolist()], dtype=np.float64)
    a = (slice(NG, NG + nx), slice(NG, NG + ny), slice(NG, NG + nz))
    H[(0,) + a] = rho
    H[(1,) + a] = 0.0
    H[(2,) + a] = 0.0
    H[(3,) + a] = 0.0
    H[(4,) + a] = P / (gamma - 1.0)
    _store(U, H)
    return rho_c, r_scale, K, r_core


def thermal_bomb(U, nx, ny, nz, dx, dy, dz, *, E_SN, r_bomb, r_bomb_inner=0.0, x0=0.0, y0=0.0, z0=0.0,
                 x_center=0.0, y_center=0.0, z_center=0.0, bipolar_theta_deg=180.0):
    """thermal_bomb! (src/stellar_ic.jl:210-253): E_SN deposited as thermal
    energy, mass-weighted over the cells of the shell r_bomb_inner <= r <
    r_bomb (within the polar cones of half angle bipolar_theta_deg).
    Returns M_bomb; raises ValueError when the shell holds no gas."""
    H = _read(U, nx, ny, nz)
    dV = float(dx) * float(dy) * float(dz)
    rin2, rout2 = float(r_bomb_inner) ** 2, float(r_bomb) ** 2
    mu_min = math.cos(float(bipolar_theta_deg) * math.pi / 180.0)
    xc = x0 + (np.arange(1, nx + 1, dtype=np.float64) - 0.5) * dx - x_center
    yc = y0 + (np.arange(1, ny + 1, dtype=np.float64) - 0.5) * dy - y_center
    zc = z0 + (np.arange(1, nz + 1, dtype=np.float64) - 0.5) * dz - z_center
    r2 = _r2(xc, yc, zc)
    in_shell = (rin2 <= r2) & (r2 < rout2)
    in_cone = np.where(r2 <= 0.0, True, np.abs(zc)[None, None, :] >= np.sqrt(r2) * mu_min)
    sel = in_shell & in_cone
    a = (slice(NG, NG + nx), slice(NG, NG + ny), slice(NG, NG + nz))
    rho = H[(0,) + a]
    M_bomb = _seq_sum((rho * dV).ravel(order="F")[sel.ravel(order="F")])
    if not M_bomb > 0.0:
        raise ValueError(f"thermal_bomb: no gas in shell [{r_bomb_inner}, {r_bomb}) within cone "
                         f"theta_j={bipolar_theta_deg} deg")
    fac = float(E_SN) / M_bomb
    E = H[(4,) + a]
    H[(4,) + a] = np.where(sel, E + fac * rho, E)
    _store(U, H)
    return M_bomb


def apply_stellar_rotation(U, nx, ny, nz, dx, gamma, Omega, *, v_star_y=0.0, x_star=0.0, y_star=0.0, rho_thresh,
                           x0=0.0, y0=0.0):
    """apply_stellar_rotation! (scripts/run_sn50_fiducial.jl:421-446): the
    gas of every active cell with rho > rho_thresh takes the velocity
    v = (0, v_star_y, 0) + Omega z x (r - r_star); its internal energy
    (U[4] holds only internal energy before the overlay) is kept and the
    kinetic energy added.  x0, y0: lower corner of the grid; dx the cell width
    the reference uses on both axes."""
    H = _read(U, nx, ny, nz)
    a = (slice(NG, NG + nx), slice(NG, NG + ny), slice(NG, NG + nz))
    rho = H[(0,) + a]
    sel = rho > rho_thresh
    xc = x0 + (np.arange(1, nx + 1, dtype=np.float64) - 0.5) * dx - x_star
    yc = y0 + (np.arange(1, ny + 1, dtype=np.float64) - 0.5) * dx - y_star
    shape = (nx, ny, nz)
    vx = np.broadcast_to(-Omega * yc[None, :, None], shape)
    vy = np.broadcast_to(v_star_y + Omega * xc[:, None, None], shape)
    vz = np.zeros(shape)
    P_int = H[(4,) + a] * (gamma - 1.0)
    ke = ((vx * vx + vy * vy) + vz * vz)
    m = {1: rho * vx, 2: rho * vy, 3: rho * vz}
    for q in (1, 2, 3):
        H[(q,) + a] = np.where(sel, m[q], H[(q,) + a])
    H[(4,) + a] = np.where(sel, P_int / (gamma - 1.0) + 0.5 * rho * ke, H[(4,) + a])
    if H is not U:
        _store(U, H)
