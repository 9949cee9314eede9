"""Checkpoints, snapshots and BH trajectories in the reference's HDF5 layouts
(src/checkpoint.jl, src/io.jl) through libbsn's own HDF5 writer and reader
(include/bsn.h: no HDF5 library is linked).

State arrays are CUDA float64 tensors in the reference layout U[q,i,j,k]
(`bsn.state`) or Fortran-ordered numpy arrays of the same shape (host); BHs
are `bsn.BlackHole` records, updated or created as the reference's functions
do.  Names and return values follow the reference's functions."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

from . import api
from ._lib import BSNError, bsn_bh, bsn_ckpt_meta, bsn_fmr2, bsn_grid_meta, load

__all__ = ["save_checkpoint_uniform", "checkpoint_wait", "load_checkpoint_uniform", "save_checkpoint",
           "load_checkpoint", "write_snapshot", "read_snapshot", "init_trajectory_file", "append_trajectory",
           "read_trajectory"]

NG = api.NG


def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


def _state_arg(U, nx, ny, nz):
    """(ctx, pointer, on_device) of a device tensor or host array in the state layout."""
    shape = (5, nx + 2 * NG, ny + 2 * NG, nz + 2 * NG)
    if isinstance(U, torch.Tensor):
        api._check_state(U, nx, ny, nz)
        return api.context(), api._ptr(U), 1
    if not (isinstance(U, np.ndarray) and U.dtype == np.float64 and U.shape == shape and U.flags.f_contiguous):
        raise TypeError(f"U must be a CUDA state tensor or a Fortran-ordered float64 array of shape {shape}")
    return None, C.c_void_p(U.ctypes.data), 0


def _check(rc, what, ctx=None):
    if rc != 0:
        msg = load().bsn_last_error(ctx).decode() if ctx is not None else what
        raise BSNError(rc, msg)


def save_checkpoint_uniform(path, U, bhs, *, t, step, dt_last, t_snap, t_bh2_sink_on, nx, ny, nz, dx, dy, dz, gamma,
                            x0, y0, z0, rho_floor, P_floor, asynchronous=False):
    """save_checkpoint_uniform (src/checkpoint.jl:222-265).  With
    asynchronous=True (device U only) the state is copied on the current
    stream and written in the background; `checkpoint_wait()` finishes it."""
    ctx, p, dev = _state_arg(U, nx, ny, nz)
    arr = api._bh_array(bhs)
    g = bsn_grid_meta(nx, ny, nz, dx, dy, dz, gamma, x0, y0, z0, rho_floor, P_floor)
    m = bsn_ckpt_meta(float(t), int(step), float(dt_last), float(t_snap), float(t_bh2_sink_on))
    L = load()
    if asynchronous:
        if not dev:
            raise TypeError("asynchronous checkpoints take a device state")
        _check(L.bsn_save_checkpoint_uniform_async(ctx, _path(path), p, arr, len(bhs), C.byref(g), C.byref(m)),
               "save_checkpoint_uniform", ctx)
        return path
    _check(L.bsn_save_checkpoint_uniform(ctx, _path(path), p, dev, arr, len(bhs), C.byref(g), C.byref(m)),
           "save_checkpoint_uniform", ctx)
    return path


def checkpoint_wait():
    """Finish the context's asynchronous checkpoint (if any); raises its error."""
    ctx = api.context()
    _check(load().bsn_checkpoint_wait(ctx), "checkpoint_wait", ctx)


def load_checkpoint_uniform(path, *, device="cuda"):
    """load_checkpoint_uniform (src/checkpoint.jl:277-318) -> (U, bhs, grid,
    meta); U on `device` ("cpu": a Fortran-ordered numpy array)."""
    L = load()
    g, m, nb = bsn_grid_meta(), bsn_ckpt_meta(), C.c_int(0)
    _check(L.bsn_load_checkpoint_uniform(None, _path(path), None, 0, None, 0, C.byref(nb), C.byref(g), C.byref(m)),
           f"load_checkpoint_uniform({path})")
    arr = (bsn_bh * max(1, nb.value))()
    if device == "cpu":
        U = np.zeros((5, g.nx + 2 * NG, g.ny + 2 * NG, g.nz + 2 * NG), order="F")
        ctx, p, dev = None, C.c_void_p(U.ctypes.data), 0
    else:
        U = api.state(g.nx, g.ny, g.nz, device=device)
        ctx, p, dev = api.context(), api._ptr(U), 1
    _check(L.bsn_load_checkpoint_uniform(ctx, _path(path), p, dev, arr, nb.value, C.byref(nb), C.byref(g),
                                         C.byref(m)), f"load_checkpoint_uniform({path})", ctx)
    bhs = [bsn_bh.from_buffer_copy(arr[i]) for i in range(nb.value)]
    grid = dict(nx=g.nx, ny=g.ny, nz=g.nz, dx=g.dx, dy=g.dy, dz=g.dz, gamma=g.gamma, x0=g.x0, y0=g.y0, z0=g.z0,
                rho_floor=g.rho_floor, P_floor=g.P_floor)
    meta = dict(t=m.t, step=m.step, dt_last=m.dt_last, t_snap=m.t_snap, t_bh2_sink_on=m.t_bh2_sink_on,
                format_version=1)
    return U, bhs, grid, meta


def save_checkpoint(path, G, bhs, *, t=0.0, step=0, dt_last=0.0):
    """save_checkpoint (src/checkpoint.jl:39-100) of a two-level
    `bsn.FMRGrid3D` on the device."""
    ctx = api.context()
    arr = api._bh_array(bhs)
    _check(load().bsn_save_checkpoint_fmr(ctx, _path(path), C.byref(G.s), 1, arr, len(bhs), float(t), int(step),
                                          float(dt_last)), "save_checkpoint", ctx)
    return path


def load_checkpoint(path, *, device="cuda"):
    """load_checkpoint (src/checkpoint.jl:101-165) -> (G, bhs, meta): a
    `bsn.FMRGrid3D` with the saved coarse and fine states (the fine level as
    saved, not re-prolonged)."""
    L = load()
    s = bsn_fmr2()
    nb, t, dt_last, step = C.c_int(0), C.c_double(0), C.c_double(0), C.c_longlong(0)
    _check(L.bsn_load_checkpoint_fmr(None, _path(path), C.byref(s), 0, None, 0, C.byref(nb), C.byref(t),
                                     C.byref(step), C.byref(dt_last)), f"load_checkpoint({path})")
    Uc = api.state(s.ncx, s.ncy, s.ncz, device=device)
    bc = "periodic" if s.bc == 1 else "outflow"
    G = api.FMRGrid3D(Uc, s.ncx, s.ncy, s.ncz, s.dxc, s.ci_lo, s.ci_hi, s.cj_lo, s.cj_hi, s.ck_lo, s.ck_hi, s.ratio,
                      s.gamma, bc=bc, rho_floor=s.rho_floor, P_floor=s.P_floor, dyc=s.dyc, dzc=s.dzc, init=False)
    if G.fine_dims != (s.nfx, s.nfy, s.nfz):
        raise BSNError(7, f"{path}: fine level {(s.nfx, s.nfy, s.nfz)} does not match the refined box")
    arr = (bsn_bh * max(1, nb.value))()
    ctx = api.context()
    _check(L.bsn_load_checkpoint_fmr(ctx, _path(path), C.byref(G.s), 1, arr, nb.value, C.byref(nb), C.byref(t),
                                     C.byref(step), C.byref(dt_last)), f"load_checkpoint({path})", ctx)
    bhs = [bsn_bh.from_buffer_copy(arr[i]) for i in range(nb.value)]
    return G, bhs, dict(t=t.value, step=step.value, dt_last=dt_last.value, format_version=1)


def write_snapshot(filename, U, nx, ny, nz, dx, dy, dz, t, gamma):
    """write_snapshot (src/io.jl:29-52): the active cells' five fields."""
    ctx, p, dev = _state_arg(U, nx, ny, nz)
    _check(load().bsn_write_snapshot(ctx, _path(filename), p, dev, nx, ny, nz, float(dx), float(dy), float(dz),
                                     float(t), float(gamma)), "write_snapshot", ctx)


def read_snapshot(filename):
    """read_snapshot (src/io.jl:54-83) -> (U_active[q,i,j,k], nx, ny, nz, dx,
    dy, dz, t, gamma), U_active a Fortran-ordered numpy array."""
    L = load()
    n = [C.c_int(0) for _ in range(3)]
    f = [C.c_double(0) for _ in range(5)]
    args = [C.byref(v) for v in n] + [C.byref(v) for v in f]
    _check(L.bsn_read_snapshot(_path(filename), None, 0, *args), f"read_snapshot({filename})")
    nx, ny, nz = (v.value for v in n)
    U = np.zeros((5, nx, ny, nz), order="F")
    _check(L.bsn_read_snapshot(_path(filename), U.ctypes.data_as(C.POINTER(C.c_double)), U.size, *args),
           f"read_snapshot({filename})")
    dx, dy, dz, t, g = (v.value for v in f)
    return U, nx, ny, nz, dx, dy, dz, t, g


def init_trajectory_file(filename, n_bh):
    """init_trajectory_file (src/io.jl:96-118)."""
    _check(load().bsn_trajectory_init(_path(filename), int(n_bh)), "init_trajectory_file")


def append_trajectory(filename, t, bhs):
    """append_trajectory (src/io.jl:120-142): one record for all BHs."""
    arr = api._bh_array(bhs)
    _check(load().bsn_trajectory_append(_path(filename), float(t), arr, len(bhs)), "append_trajectory")


def read_trajectory(filename):
    """read_trajectory (src/io.jl:144-180) -> (t, [{mass, pos, vel, rsink}])
    with pos/vel of shape (N, 3)."""
    L = load()
    nd, nb = C.c_int(0), C.c_int(0)
    _check(L.bsn_trajectory_read(_path(filename), C.byref(nd), C.byref(nb), None, None, None, None, None, 0),
           "read_trajectory")
    N, B = nd.value, nb.value
    t = np.zeros(max(N, 1))
    mass, rs = np.zeros(max(B * N, 1)), np.zeros(max(B * N, 1))
    pos, vel = np.zeros(max(3 * B * N, 1)), np.zeros(max(3 * B * N, 1))
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    _check(L.bsn_trajectory_read(_path(filename), C.byref(nd), C.byref(nb), ptr(t), ptr(mass), ptr(pos), ptr(vel),
                                 ptr(rs), N), "read_trajectory")
    out = []
    for b in range(B):
        out.append(dict(mass=mass[b * N:(b + 1) * N].copy(), rsink=rs[b * N:(b + 1) * N].copy(),
                        pos=pos[3 * b * N:3 * (b + 1) * N].reshape(N, 3).copy(),
                        vel=vel[3 * b * N:3 * (b + 1) * N].reshape(N, 3).copy()))
    return t[:N].copy(), out
