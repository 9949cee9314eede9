"""Reference-named entry points over libbsn (FP64 parity path).

Array conventions (the reference's Julia layout, column-major):
  * state U: torch.float64 CUDA tensor of shape (5, nx+6, ny+6, nz+6) with
    strides (1, 5, 5*(nx+6), 5*(nx+6)*(ny+6)) -- `state()` makes one, and
    `torch.from_numpy(fortran_array).cuda()` keeps these strides.
  * flux arrays: shapes (5,NXT+1,NYT,NZT), (5,NXT,NYT+1,NZT), (5,NXT,NYT,NZT+1).
  * potentials/densities on the active grid: shape (nx, ny, nz), strides
    (1, nx, nx*ny).
Errors raise BSNError (the reference throws on bad input).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Sequence

import numpy as np
import torch

from ._lib import BSNError, bsn_bh, bsn_fmr2, bsn_stage_sources, load

NG = 3
BC = {"outflow": 0, "periodic": 1}

__all__ = [
    "NG", "BSNError", "BlackHole", "state", "flux_arrays", "active_grid", "context", "launch_count",
    "fill_ghost_3d_outflow", "fill_ghost_3d_periodic", "apply_floors_3d", "euler3d_rhs", "euler3d_step",
    "cfl_dt_3d", "add_bh_gravity_source", "gas_force_on_bh", "add_sink_sources", "accrete", "r_sink", "t_sink",
    "nbody_step", "KeplerOrbit", "kepler_update", "solve_poisson_isolated", "add_self_gravity_source",
    "poisson_slab_forward", "poisson_slab_zconv", "poisson_slab_inverse",
    "apply_sg_force_level", "apply_sg_force_slab", "coupled_step", "FMRGrid3D", "fmr3d_step", "cfl_dt_fmr3d", "solve_fmr_poisson",
    "restrict_density_to_coarse", "FMRHierarchy3D", "fmr_nested_step", "cfl_dt_fmr_nested",
    "fmr_nested_run_steps", "coupled_nested_run_steps", "rotating_frame_source", "relax_damping_source",
    "relax_ic", "DIAG_FIELDS", "DIAG_RECORD", "set_tma", "get_tma", "get_tile_tma", "set_stiff_guard",
]

# ---------------------------------------------------------------------------
# context / stream plumbing

_ctx = {}


def context(device: int | None = None) -> C.c_void_p:
    """The library context of a CUDA device (created once per device)."""
    if not torch.cuda.is_available():
        raise RuntimeError("bsn needs a CUDA device (sm_100a); no CPU fallback exists")
    dev = torch.cuda.current_device() if device is None else int(device)
    if dev not in _ctx:
        L = load()
        h = C.c_void_p()
        rc = L.bsn_ctx_create(C.byref(h), dev, None)
        if rc != 0:
            raise BSNError(rc, f"bsn_ctx_create(device={dev}) failed")
        _ctx[dev] = h
    h = _ctx[dev]
    load().bsn_ctx_set_stream(h, C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    return h


def launch_count(device: int | None = None) -> int:
    """Kernels this process's context has launched on `device`."""
    return int(load().bsn_ctx_launch_count(context(device)))


def _call(name: str, *args):
    L = load()
    rc = getattr(L, name)(*args)
    if rc != 0:
        msg = L.bsn_last_error(args[0]).decode() if args and isinstance(args[0], C.c_void_p) else name
        raise BSNError(rc, msg)


def _ptr(t) -> C.c_void_p | None:
    if t is None:
        return None
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64):
        raise TypeError("expected a CUDA float64 tensor")
    return C.c_void_p(t.data_ptr())


def _cptr(t) -> C.c_void_p:
    """a CUDA complex128 tensor as interleaved doubles"""
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.complex128):
        raise TypeError("expected a CUDA complex128 tensor")
    return C.c_void_p(t.data_ptr())


def _check_state(U: torch.Tensor, nx: int, ny: int, nz: int, name="U"):
    want = (5, nx + 2 * NG, ny + 2 * NG, nz + 2 * NG)
    if tuple(U.shape) != want:
        raise ValueError(f"{name} has shape {tuple(U.shape)}, expected {want}")
    X, Y = nx + 2 * NG, ny + 2 * NG
    if U.stride() != (1, 5, 5 * X, 5 * X * Y):
        raise ValueError(f"{name} must use the reference column-major layout (strides {U.stride()})")


def _check_grid(a: torch.Tensor, nx: int, ny: int, nz: int, name: str):
    if tuple(a.shape) != (nx, ny, nz) or a.stride() != (1, nx, nx * ny):
        raise ValueError(f"{name} must be a column-major (nx,ny,nz) array")


def state(nx: int, ny: int, nz: int, device="cuda", dtype=torch.float64) -> torch.Tensor:
    """Zeroed state array U[q,i,j,k] of the reference (5, nx+6, ny+6, nz+6)."""
    X, Y, Z = nx + 2 * NG, ny + 2 * NG, nz + 2 * NG
    return torch.zeros((Z, Y, X, 5), device=device, dtype=dtype).permute(3, 2, 1, 0)


def flux_arrays(nx: int, ny: int, nz: int, device="cuda"):
    X, Y, Z = nx + 2 * NG, ny + 2 * NG, nz + 2 * NG
    mk = lambda a, b, c: torch.zeros((c, b, a, 5), device=device, dtype=torch.float64).permute(3, 2, 1, 0)
    return mk(X + 1, Y, Z), mk(X, Y + 1, Z), mk(X, Y, Z + 1)


def active_grid(nx: int, ny: int, nz: int, device="cuda") -> torch.Tensor:
    return torch.zeros((nz, ny, nx), device=device, dtype=torch.float64).permute(2, 1, 0)


# ---------------------------------------------------------------------------
# black holes (src/BinarySupernova.jl:130-171)

def BlackHole(pos, vel, mass, eps, c_code, r_floor) -> bsn_bh:
    return bsn_bh((C.c_double * 3)(*pos), (C.c_double * 3)(*vel), float(mass), float(eps), float(c_code),
                  float(r_floor))


def _bh_array(bhs: Sequence[bsn_bh]):
    arr = (bsn_bh * max(1, len(bhs)))()
    for i, b in enumerate(bhs):
        arr[i] = b
    return arr


def _bh_writeback(bhs, arr):
    for i, b in enumerate(bhs):
        C.memmove(C.addressof(b), C.addressof(arr[i]), C.sizeof(bsn_bh))


def r_sink(bh: bsn_bh) -> float:
    """src/BinarySupernova.jl:159"""
    v = 6.0 * bh.mass / bh.c_code ** 2
    return v if v > bh.r_floor else bh.r_floor


def t_sink(bh: bsn_bh, f_sink: float = 1.0) -> float:
    """src/BinarySupernova.jl:167-171"""
    rs = r_sink(bh)
    return f_sink * rs / math.sqrt(2.0 * bh.mass / rs)


# ---------------------------------------------------------------------------
# src/euler3d.jl

def fill_ghost_3d_outflow(U, nx, ny, nz):
    _check_state(U, nx, ny, nz)
    _call("bsn_fill_ghost_3d_f64", context(), _ptr(U), nx, ny, nz, 0)


def fill_ghost_3d_periodic(U, nx, ny, nz):
    _check_state(U, nx, ny, nz)
    _call("bsn_fill_ghost_3d_f64", context(), _ptr(U), nx, ny, nz, 1)


def apply_floors_3d(U, nx, ny, nz, rho_floor, P_floor, gamma):
    _check_state(U, nx, ny, nz)
    _call("bsn_apply_floors_3d_f64", context(), _ptr(U), nx, ny, nz, float(rho_floor), float(P_floor), float(gamma))


def euler3d_rhs(dU, Fx, Fy, Fz, U, nx, ny, nz, dx, dy, dz, gamma, *, bc="outflow", rho_floor=0.0, P_floor=0.0,
                fill_ghosts=True):
    _check_state(U, nx, ny, nz)
    _check_state(dU, nx, ny, nz, "dU")
    _call("bsn_euler3d_rhs_f64", context(), _ptr(dU), _ptr(Fx), _ptr(Fy), _ptr(Fz), _ptr(U), nx, ny, nz,
          float(dx), float(dy), float(dz), float(gamma), BC[bc], float(rho_floor), float(P_floor), int(fill_ghosts))


def euler3d_rhs_f32(dU, Fx, Fy, Fz, U, nx, ny, nz, dx, dy, dz, gamma, *, bc="outflow", rho_floor=0.0, P_floor=0.0,
                    fill_ghosts=True):
    """euler3d_rhs! with the FP32 stencils (src/euler3d.jl:182-205): face
    fluxes from the FP32 reconstruction and HLLC (stiff faces in FP64 when the
    context's stiff guard is on), stored as FP32 values; divergence in FP64."""
    _check_state(U, nx, ny, nz)
    _check_state(dU, nx, ny, nz, "dU")
    _call("bsn_euler3d_rhs_f32", context(), _ptr(dU), _ptr(Fx), _ptr(Fy), _ptr(Fz), _ptr(U), nx, ny, nz,
          float(dx), float(dy), float(dz), float(gamma), BC[bc], float(rho_floor), float(P_floor), int(fill_ghosts))


def euler3d_step(U, nx, ny, nz, dx, dy, dz, dt, gamma, *, bc="outflow", rho_floor=0.0, P_floor=0.0):
    _check_state(U, nx, ny, nz)
    _call("bsn_euler3d_step_f64", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz), float(dt),
          float(gamma), BC[bc], float(rho_floor), float(P_floor))


def cfl_dt_3d(U, nx, ny, nz, dx, dy, dz, gamma, cfl) -> float:
    _check_state(U, nx, ny, nz)
    out = C.c_double()
    _call("bsn_cfl_dt_3d_f64", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz), float(gamma),
          float(cfl), C.byref(out))
    return out.value


# ---------------------------------------------------------------------------
# src/gravity_bh.jl, src/sinks.jl, src/nbody.jl, src/kepler_orbit.jl

def add_bh_gravity_source(dU, U, nx, ny, nz, dx, dy, dz, bhs, x0, y0, z0):
    arr = _bh_array(bhs)
    _call("bsn_add_bh_gravity_source_f64", context(), _ptr(dU), _ptr(U), nx, ny, nz, float(dx), float(dy),
          float(dz), arr, len(bhs), float(x0), float(y0), float(z0))


def gas_force_on_bh(U, nx, ny, nz, dx, dy, dz, bh, x0, y0, z0) -> np.ndarray:
    out = (C.c_double * 3)()
    _call("bsn_gas_force_on_bh_f64", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz),
          C.byref(bh), float(x0), float(y0), float(z0), out)
    return np.array(out[:])


def add_sink_sources(dU, U, nx, ny, nz, dx, dy, dz, bhs, x0, y0, z0, *, f_sink=1.0, torque_free=True,
                     rho_sink_min=0.0):
    arr = _bh_array(bhs)
    _call("bsn_add_sink_sources_f64", context(), _ptr(dU), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz),
          arr, len(bhs), float(x0), float(y0), float(z0), float(f_sink), int(bool(torque_free)),
          float(rho_sink_min))


def accrete(bh, U, nx, ny, nz, dx, dy, dz, x0, y0, z0, dt, *, f_sink=1.0, rho_sink_min=0.0):
    _call("bsn_accrete_f64", context(), C.byref(bh), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz),
          float(x0), float(y0), float(z0), float(dt), float(f_sink), float(rho_sink_min))


def add_bh_gravity_source_slab(dU, U, nx, ny, nz, dx, dy, dz, bhs, x0, y0, z0, k0):
    """add_bh_gravity_source! on a z-slab whose first active plane is global plane k0."""
    arr = _bh_array(bhs)
    _call("bsn_add_bh_gravity_source_slab_f64", context(), _ptr(dU), _ptr(U), nx, ny, nz, float(dx), float(dy),
          float(dz), arr, len(bhs), float(x0), float(y0), float(z0), int(k0))


def add_sink_sources_slab(dU, U, nx, ny, nz, dx, dy, dz, bhs, x0, y0, z0, k0, *, f_sink=1.0, torque_free=True,
                          rho_sink_min=0.0):
    """add_sink_sources! on a z-slab whose first active plane is global plane k0."""
    arr = _bh_array(bhs)
    _call("bsn_add_sink_sources_slab_f64", context(), _ptr(dU), _ptr(U), nx, ny, nz, float(dx), float(dy),
          float(dz), arr, len(bhs), float(x0), float(y0), float(z0), float(f_sink), int(bool(torque_free)),
          float(rho_sink_min), int(k0))


def gas_force_pairs_slab(U, nx, ny, nz, dx, dy, dz, bh, x0, y0, z0, k0) -> np.ndarray:
    """The slab's compensated gas_force_on_bh partial sums: (hi, lo) per component, shape (6,)."""
    out = (C.c_double * 6)()
    _call("bsn_gas_force_on_bh_slab_f64", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz),
          C.byref(bh), float(x0), float(y0), float(z0), int(k0), out)
    return np.array(out[:])


def merge_force_pairs(pairs) -> np.ndarray:
    """Merge per-slab (hi, lo) pairs (rows in rank order) into the force (host)."""
    P = np.ascontiguousarray(np.asarray(pairs, dtype=np.float64).reshape(-1, 6))
    out = (C.c_double * 3)()
    rc = load().bsn_merge_force_pairs(P.ctypes.data_as(C.POINTER(C.c_double)), P.shape[0], out)
    if rc != 0:
        raise BSNError(rc, "merge_force_pairs")
    return np.array(out[:])


def sink_box(bh, nx, ny, nz, dx, dy, dz, x0, y0, z0):
    """The global active box {ilo, ihi, jlo, jhi, klo, khi} that holds the sink sphere (host)."""
    b = (C.c_int * 6)()
    rc = load().bsn_sink_box(C.byref(bh), nx, ny, nz, float(dx), float(dy), float(dz), float(x0), float(y0),
                             float(z0), b)
    if rc != 0:
        raise BSNError(rc, "sink_box")
    return tuple(b[:])


def sink_terms_slab(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, k0, bh, dt, box, *, f_sink=1.0, rho_sink_min=0.0):
    """accrete!'s terms over this slab's part of the global box, (n, 4) host array in (k, j, i) order."""
    ilo, ihi, jlo, jhi, klo, khi = box
    kl, kh = max(klo, k0), min(khi, k0 + nz - 1)
    cap = max(0, ihi - ilo + 1) * max(0, jhi - jlo + 1) * max(0, kh - kl + 1)
    out = np.zeros((max(cap, 1), 4))
    n = C.c_longlong(0)
    b = (C.c_int * 6)(*box)
    _call("bsn_sink_terms_slab_f64", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz), float(x0),
          float(y0), float(z0), int(k0), C.byref(bh), float(dt), float(f_sink), float(rho_sink_min), b,
          out.ctypes.data_as(C.POINTER(C.c_double)), cap, C.byref(n))
    return out[:n.value]


def euler3d_stage(Uout, Uin, Un, nx, ny, nz, dx, dy, dz, dt, gamma, stage, *, rho_floor=0.0, P_floor=0.0,
                  precision="f64", bhs=(), nsink=0, f_sink=1.0, torque_free=True, rho_sink_min=0.0, x0=0.0,
                  y0=0.0, z0=0.0, k0=0, phi=None, phi_lo=None, phi_hi=None):
    """One SSP-RK3 stage (1, 2 or 3) of euler3d_step! / coupled_step! in one
    fused launch, with Uin's ghost cells as the caller left them; Uout must
    differ from Uin, and stage 1 takes Un = Uin.  Sources: BH gravity of
    `bhs`, the sinks of bhs[:nsink], the self-gravity gradient of `phi` (the
    potential of Uin's floored density) with the neighbouring slabs' planes
    phi_lo / phi_hi; k0 is the slab's first global plane."""
    for a, name in ((Uout, "Uout"), (Uin, "Uin"), (Un, "Un")):
        _check_state(a, nx, ny, nz, name)
    arr = _bh_array(bhs)
    src = bsn_stage_sources(arr, len(bhs), int(nsink), float(f_sink), int(bool(torque_free)), float(rho_sink_min),
                            float(x0), float(y0), float(z0), int(k0),
                            None if phi is None else phi.data_ptr(),
                            None if phi_lo is None else phi_lo.data_ptr(),
                            None if phi_hi is None else phi_hi.data_ptr())
    _call("bsn_euler3d_stage", context(), _ptr(Uout), _ptr(Uin), _ptr(Un), nx, ny, nz, float(dx), float(dy),
          float(dz), float(dt), float(gamma), int(stage), float(rho_floor), float(P_floor), PREC[precision],
          C.byref(src))


def accrete_from_terms(bh, terms):
    """The end of accrete! from the global (k, j, i)-ordered term list (host)."""
    T = np.ascontiguousarray(np.asarray(terms, dtype=np.float64).reshape(-1, 4))
    rc = load().bsn_accrete_from_terms(C.byref(bh), T.ctypes.data_as(C.POINTER(C.c_double)), T.shape[0])
    if rc != 0:
        raise BSNError(rc, "accrete_from_terms")


def nbody_step(bhs, dt, F_gas):
    arr = _bh_array(bhs)
    F = np.ascontiguousarray(np.asarray(F_gas, dtype=np.float64).reshape(-1))
    rc = load().bsn_nbody_step(arr, len(bhs), float(dt), F.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise BSNError(rc, "nbody_step")
    _bh_writeback(bhs, arr)


class KeplerOrbit:
    """src/kepler_orbit.jl:36-111 (state kept as the 13 doubles of the C ABI)."""

    def __init__(self, bhs, com=(0.0, 0.0, 0.0), nhat=None, Omega=None):
        self._st = (C.c_double * 13)()
        c = (C.c_double * 3)(*com)
        nh = None if nhat is None else (C.c_double * 3)(*nhat)
        rc = load().bsn_kepler_init(_bh_array(bhs), c, nh, -1.0 if Omega is None else float(Omega), self._st)
        if rc != 0:
            raise BSNError(rc, "KeplerOrbit: degenerate two-BH state")

    @property
    def Omega(self):
        return self._st[3]

    @property
    def com(self):
        return tuple(self._st[0:3])

    @property
    def nhat(self):
        return tuple(self._st[4:7])


def kepler_update(bhs, orbit: KeplerOrbit, t):
    arr = _bh_array(bhs)
    load().bsn_kepler_update(arr, orbit._st, float(t))
    _bh_writeback(bhs, arr)


# ---------------------------------------------------------------------------
# src/self_gravity.jl, src/fmr_gravity.jl

def solve_poisson_isolated(rho, nx, ny, nz, dx, dy, dz, *, precision="f64") -> torch.Tensor:
    """precision "f64" (the reference's arithmetic) or "f32" (FP32 transforms)."""
    _check_grid(rho, nx, ny, nz, "rho")
    phi = active_grid(nx, ny, nz, device=rho.device)
    name = {"f64": "bsn_solve_poisson_isolated_f64", "f32": "bsn_solve_poisson_isolated_f32"}[precision]
    _call(name, context(), _ptr(rho), nx, ny, nz, float(dx), float(dy), float(dz), _ptr(phi))
    return phi


def poisson_slab_forward(rho, nx, ny, nzl) -> torch.Tensor:
    """x and y transforms of a slab of nzl density planes (rho column-major
    (nx, ny, nzl)): complex128 W2 of shape (nzl, 2ny, nx+1)."""
    _check_grid(rho, nx, ny, nzl, "rho")
    W2 = torch.empty((nzl, 2 * ny, nx + 1), dtype=torch.complex128, device=rho.device)
    _call("bsn_poisson_slab_forward_f64", context(), _ptr(rho), nx, ny, nzl, _cptr(W2))
    return W2


def poisson_slab_zconv(T, nx, ny, nz, ky0, dx, dy, dz):
    """z transform, Green's function of the global nx x ny x nz grid and
    inverse z transform of T (complex128 (nz, nky, nx+1), ky = ky0 + kyl), in place."""
    if T.dtype != torch.complex128 or T.dim() != 3 or T.shape[0] != nz or T.shape[2] != nx + 1 \
            or not T.is_contiguous():
        raise ValueError(f"T must be contiguous complex128 (nz, nky, nx+1), got {tuple(T.shape)} {T.dtype}")
    _call("bsn_poisson_slab_zconv_f64", context(), _cptr(T), nx, ny, nz, int(ky0), int(T.shape[1]), float(dx),
          float(dy), float(dz))


def poisson_slab_inverse(W2, nx, ny, nzl) -> torch.Tensor:
    """y and x inverse transforms of W2 (complex128 (nzl, 2ny, nx+1)): the
    slab's potential, column-major (nx, ny, nzl)."""
    if W2.dtype != torch.complex128 or tuple(W2.shape) != (nzl, 2 * ny, nx + 1) or not W2.is_contiguous():
        raise ValueError(f"W2 must be contiguous complex128 {(nzl, 2 * ny, nx + 1)}, got {tuple(W2.shape)}")
    phi = active_grid(nx, ny, nzl, device=W2.device)
    _call("bsn_poisson_slab_inverse_f64", context(), _cptr(W2), nx, ny, nzl, _ptr(phi))
    return phi


def apply_sg_force_level(dU, U, phi, nx, ny, nz, dx, dy, dz):
    """_apply_sg_force_level! (src/fmr_gravity.jl:146-156)."""
    _check_grid(phi, nx, ny, nz, "phi")
    _call("bsn_sg_gradient_f64", context(), _ptr(dU), _ptr(U), _ptr(phi), nx, ny, nz, float(dx), float(dy),
          float(dz))


def apply_sg_force_slab(dU, U, phi, nx, ny, nz, dx, dy, dz, phi_lo=None, phi_hi=None):
    """_apply_sg_force_level! on a z-slab of a larger grid: phi_lo / phi_hi
    are the (nx, ny) planes of Phi just below / above the slab (None at the
    larger grid's own z boundary)."""
    _check_grid(phi, nx, ny, nz, "phi")
    for p in (phi_lo, phi_hi):
        if p is not None and not (p.is_contiguous() and p.numel() == nx * ny):
            raise ValueError("neighbour planes of Phi must be contiguous (nx, ny) arrays")
    _call("bsn_sg_gradient_slab_f64", context(), _ptr(dU), _ptr(U), _ptr(phi), _ptr(phi_lo), _ptr(phi_hi), nx, ny,
          nz, float(dx), float(dy), float(dz))


def add_self_gravity_source(dU, U, nx, ny, nz, dx, dy, dz):
    _call("bsn_add_self_gravity_source_f64", context(), _ptr(dU), _ptr(U), nx, ny, nz, float(dx), float(dy),
          float(dz))


# ---------------------------------------------------------------------------
# scripts/run_sn50_fiducial.jl:756-818

def coupled_step(U, bhs, dt, t, nx, ny, nz, dx, x0, y0, z0, gamma, f_sink, rho_floor, P_floor, torque_free,
                 self_gravity, t_bh2_sink_on, rho_sink_min, evolve_orbit=True):
    """One production step; returns F_gas (nbh x 3).  `bhs` is updated in place."""
    arr = _bh_array(bhs)
    Fg = (C.c_double * (3 * max(1, len(bhs))))()
    _call("bsn_coupled_step_f64", context(), _ptr(U), arr, len(bhs), float(dt), float(t), nx, ny, nz, float(dx),
          float(x0), float(y0), float(z0), float(gamma), float(f_sink), float(rho_floor), float(P_floor),
          int(bool(torque_free)), int(bool(self_gravity)), float(t_bh2_sink_on), float(rho_sink_min),
          int(bool(evolve_orbit)), Fg)
    _bh_writeback(bhs, arr)
    return np.array(Fg[: 3 * len(bhs)]).reshape(len(bhs), 3)


# The per-step record of the device driver loops (coupled_run_steps,
# coupled_nested_run_steps): t, dt, the driver's diagnostics, and the mass
# ledger since the start of the call -- mass added by the floors, mass that
# left through the domain boundary, mass the sink sources drained from the
# gas, mass accrete! credited to the BHs.  The gas mass closes as
#   M_gas(t) = M_gas(0) + floors_in - outflow - drained
# and the BHs gain `accreted`, which accrete! takes from the end-of-step
# state while the sources drain the gas stage by stage (src/sinks.jl:74-109
# against src/gpu_kernels.jl:238-284): accreted - drained is the reference's
# own bookkeeping difference, not a loss of the update.
DIAG_FIELDS = ("t", "dt", "E_gas", "KE_gas", "Px", "Py", "Pz", "Lx", "Ly", "Lz", "M_bound", "M_gas",
               "floors_in", "outflow", "drained", "accreted")
DIAG_RECORD = len(DIAG_FIELDS)


def _check_diag(diag):
    if diag is not None and not (diag.is_cuda and diag.dtype == torch.float64 and diag.is_contiguous()
                                 and diag.dim() == 2 and diag.shape[1] == DIAG_RECORD):
        raise TypeError(f"diag must be a contiguous CUDA float64 tensor of shape (cap, {DIAG_RECORD})")


def coupled_run_steps(U, bhs, nx, ny, nz, dx, x0, y0, z0, gamma, cfl, *, n_steps, t=0.0, t_end=0.0, dt_max=0.0,
                      f_sink=1.0, rho_floor=0.0, P_floor=0.0, torque_free=True, self_gravity=False,
                      t_bh2_sink_on=0.0, rho_sink_min=0.0, evolve_orbit=True, precision="f64", diag=None):
    """The coupled_step! driver loop on the device (one CUDA graph per step);
    returns (t, steps) and updates `bhs` in place.  diag: optional CUDA float64
    tensor (cap, DIAG_RECORD) receiving after every step the record
    {t, dt, diagnostics(...) [10 values], mass ledger [4 values]} (see
    DIAG_FIELDS; the ledger totals count from the start of this call)."""
    _check_state(U, nx, ny, nz)
    _check_diag(diag)
    arr = _bh_array(bhs)
    tt = C.c_double(float(t))
    nd = C.c_int(0)
    _call("bsn_coupled_run_steps", context(), _ptr(U), arr, len(bhs), nx, ny, nz, float(dx), float(x0), float(y0),
          float(z0), float(gamma), float(cfl), float(dt_max), float(f_sink), float(rho_floor), float(P_floor),
          int(bool(torque_free)), int(bool(self_gravity)), float(t_bh2_sink_on), float(rho_sink_min),
          int(bool(evolve_orbit)), PREC[precision], int(n_steps), float(t_end), C.byref(tt), C.byref(nd),
          _ptr(diag) if diag is not None else None, int(diag.shape[0]) if diag is not None else 0)
    _bh_writeback(bhs, arr)
    return tt.value, nd.value


def rotating_frame_source(dU, U, nx, ny, nz, dx, dy, dz, x0, y0, z0, Omega):
    """rotating_frame_source! (src/relax_ic.jl:150-176)."""
    _check_state(U, nx, ny, nz)
    _check_state(dU, nx, ny, nz, "dU")
    _call("bsn_rotating_frame_source_f64", context(), _ptr(dU), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz),
          float(x0), float(y0), float(z0), float(Omega))


def relax_damping_source(dU, U, nx, ny, nz, dx, dy, dz, x0, y0, z0, t_damp, *, Omega=0.0):
    """relax_damping_source! (src/relax_ic.jl:59-120)."""
    _check_state(U, nx, ny, nz)
    _check_state(dU, nx, ny, nz, "dU")
    _call("bsn_relax_damping_source_f64", context(), _ptr(dU), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz),
          float(x0), float(y0), float(z0), float(t_damp), float(Omega))


def relax_ic(U, nx, ny, nz, dx, dy, dz, gamma, *, bhs=(), x0=0.0, y0=0.0, z0=0.0, t_damp=0.1, t_max=2.0, cfl=0.4,
             rho_floor=1e-10, P_floor=1e-10, KE_tol=0.01, Omega=0.0, self_gravity=False, precision="f64",
             max_steps=1000000):
    """relax_ic! (src/relax_ic.jl:200-330) on the device; returns (t, n_steps, KE_ratio)."""
    _check_state(U, nx, ny, nz)
    arr = _bh_array(list(bhs))
    t = C.c_double(0.0)
    n = C.c_int(0)
    kr = C.c_double(0.0)
    _call("bsn_relax_ic", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz), float(gamma), arr,
          len(bhs), float(x0), float(y0), float(z0), float(t_damp), float(t_max), float(cfl), float(rho_floor),
          float(P_floor), float(KE_tol), float(Omega), int(bool(self_gravity)), PREC[precision], int(max_steps),
          C.byref(t), C.byref(n), C.byref(kr))
    return t.value, n.value, kr.value


def diagnostics(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, bhs, gamma) -> np.ndarray:
    """src/diagnostics.jl totals: (E_gas, KE_gas, Px, Py, Pz, Lx, Ly, Lz, M_bound, M_gas)."""
    _check_state(U, nx, ny, nz)
    arr = _bh_array(bhs)
    out = (C.c_double * 10)()
    _call("bsn_diagnostics_f64", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz), float(x0),
          float(y0), float(z0), arr, len(bhs), float(gamma), out)
    return np.array(out[:])


# ---------------------------------------------------------------------------
# src/fmr3d.jl

class FMRGrid3D:
    """Two-level FMR grid over device level arrays (src/fmr3d.jl:109-151)."""

    def __init__(self, Uc, ncx, ncy, ncz, dxc, ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi, ratio, gamma, *,
                 bc="outflow", rho_floor=0.0, P_floor=0.0, dyc=None, dzc=None, init=True):
        _check_state(Uc, ncx, ncy, ncz, "Uc")
        dyc = dxc if dyc is None else dyc
        dzc = dxc if dzc is None else dzc
        nfx, nfy, nfz = (ci_hi - ci_lo + 1) * ratio, (cj_hi - cj_lo + 1) * ratio, (ck_hi - ck_lo + 1) * ratio
        self.Uc = Uc
        self.Uf = state(nfx, nfy, nfz, device=Uc.device)
        self.coarse_dims = (ncx, ncy, ncz)
        self.fine_dims = (nfx, nfy, nfz)
        self.s = bsn_fmr2(Uc.data_ptr(), ncx, ncy, ncz, dxc, dyc, dzc, self.Uf.data_ptr(), nfx, nfy, nfz,
                          dxc / ratio, dyc / ratio, dzc / ratio, ratio, ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi,
                          float(gamma), BC[bc], float(rho_floor), float(P_floor))
        if init:
            _call("bsn_fmr_prolong_all_f64", context(), C.byref(self.s))

    def prolong_fine_ghosts(self, Uc_src=None):
        src = self.Uc if Uc_src is None else Uc_src
        _call("bsn_fmr_prolong_fine_ghosts_f64", context(), _ptr(self.Uf), _ptr(src), C.byref(self.s))

    def restrict(self):
        _call("bsn_fmr_restrict_f64", context(), _ptr(self.Uc), _ptr(self.Uf), C.byref(self.s))

    def restrict_density_to_coarse(self):
        _call("bsn_restrict_density_to_coarse_f64", context(), C.byref(self.s))

    def prolong_scalar_trilinear(self, phic):
        """_prolong_scalar_trilinear! (src/fmr_gravity.jl:70-106): the fine
        level's potential from the coarse one (column-major active grids)."""
        _check_grid(phic, *self.coarse_dims, "phic")
        phif = active_grid(*self.fine_dims, device=phic.device)
        _call("bsn_prolong_scalar_trilinear_f64", context(), C.byref(self.s), _ptr(phic), _ptr(phif))
        return phif


def fmr3d_step(G: FMRGrid3D, dt_c, *, self_gravity=False, G_grav=1.0):
    _call("bsn_fmr3d_step_f64", context(), C.byref(G.s), float(dt_c), int(bool(self_gravity)), float(G_grav))


def cfl_dt_fmr3d(G: FMRGrid3D, cfl) -> float:
    out = C.c_double()
    _call("bsn_cfl_dt_fmr3d_f64", context(), C.byref(G.s), float(cfl), C.byref(out))
    return out.value


def fmr3d_run_steps(G: FMRGrid3D, cfl, *, n_steps, t=0.0, t_end=0.0, precision="f64", self_gravity=False,
                    G_grav=1.0):
    """Up to n_steps CFL-limited fmr3d_step!s on the device (one CUDA graph
    per step, coarse step and first fine subcycle batched); returns (t, steps)."""
    tt = C.c_double(float(t))
    nd = C.c_int(0)
    _call("bsn_fmr3d_run_steps", context(), C.byref(G.s), float(cfl), PREC[precision], int(bool(self_gravity)),
          float(G_grav), int(n_steps), float(t_end), C.byref(tt), C.byref(nd))
    return tt.value, nd.value


class FMRHierarchy3D:
    """Nested FMR levels over device arrays: a chain of FMRGrid3D pairs where
    pair k's fine level is pair k+1's coarse level (the reference's two-level
    FMRGrid3D, src/fmr3d.jl:109-151, applied pair by pair).  Each entry of
    `boxes` is (ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi, ratio) in the
    1-based active indices of the level above; levels[0] is U0."""

    def __init__(self, U0, nx, ny, nz, dx0, boxes, gamma, *, bc="outflow", rho_floor=0.0, P_floor=0.0,
                 init=True):
        if not 1 <= len(boxes) <= 3:
            raise ValueError("2 to 4 levels")
        self.pairs = []
        U, n, dx = U0, (nx, ny, nz), dx0
        for (a, b, c, d, e, f, r) in boxes:
            g = FMRGrid3D(U, *n, dx, a, b, c, d, e, f, r, gamma, bc=bc, rho_floor=rho_floor, P_floor=P_floor,
                          init=init)
            self.pairs.append(g)
            U, n, dx = g.Uf, g.fine_dims, dx / r
        self.levels = [U0] + [g.Uf for g in self.pairs]
        self.dims = [(nx, ny, nz)] + [g.fine_dims for g in self.pairs]
        self._arr = (bsn_fmr2 * len(self.pairs))(*[g.s for g in self.pairs])


def fmr_nested_step(H: FMRHierarchy3D, dt0, *, self_gravity=False, G_grav=1.0):
    _call("bsn_fmr_nested_step_f64", context(), H._arr, len(H.pairs), float(dt0), int(bool(self_gravity)),
          float(G_grav))


def cfl_dt_fmr_nested(H: FMRHierarchy3D, cfl) -> float:
    out = C.c_double()
    _call("bsn_cfl_dt_fmr_nested_f64", context(), H._arr, len(H.pairs), float(cfl), C.byref(out))
    return out.value


def fmr_nested_run_steps(H: FMRHierarchy3D, cfl, *, n_steps, t=0.0, t_end=0.0, precision="f64",
                         self_gravity=False, G_grav=1.0):
    """Up to n_steps CFL-limited nested steps on the device (one CUDA graph per
    level-0 step; each chain of first substeps batched per RK3 stage);
    returns (t, steps)."""
    tt = C.c_double(float(t))
    nd = C.c_int(0)
    _call("bsn_fmr_nested_run_steps", context(), H._arr, len(H.pairs), float(cfl), PREC[precision],
          int(bool(self_gravity)), float(G_grav), int(n_steps), float(t_end), C.byref(tt), C.byref(nd))
    return tt.value, nd.value


def coupled_nested_run_steps(H: FMRHierarchy3D, bhs, x0, y0, z0, cfl, *, n_steps, t=0.0, t_end=0.0,
                             dt_max=0.0, f_sink=1.0, torque_free=True, self_gravity=False, t_bh2_sink_on=0.0,
                             rho_sink_min=0.0, evolve_orbit=True, precision="f64", diag=None):
    """The coupled_step! driver loop on nested FMR levels, on the device (one
    CUDA graph per level-0 step); returns (t, steps) and updates `bhs` in
    place.  x0, y0, z0: lower corner of level 0.  diag: optional CUDA float64
    tensor (cap, DIAG_RECORD) receiving per step {t, dt, diagnostics of level 0,
    mass ledger of the composite grid} (see DIAG_FIELDS)."""
    _check_diag(diag)
    arr = _bh_array(bhs)
    tt = C.c_double(float(t))
    nd = C.c_int(0)
    _call("bsn_coupled_nested_run_steps", context(), H._arr, len(H.pairs), arr, len(bhs), float(x0), float(y0),
          float(z0), float(cfl), float(dt_max), float(f_sink), int(bool(torque_free)), int(bool(self_gravity)),
          float(t_bh2_sink_on), float(rho_sink_min), int(bool(evolve_orbit)), PREC[precision], int(n_steps),
          float(t_end), C.byref(tt), C.byref(nd), _ptr(diag) if diag is not None else None,
          int(diag.shape[0]) if diag is not None else 0)
    _bh_writeback(bhs, arr)
    return tt.value, nd.value


def restrict_density_to_coarse(G: FMRGrid3D):
    _call("bsn_restrict_density_to_coarse_f64", context(), C.byref(G.s))


def solve_fmr_poisson(G: FMRGrid3D):
    phic = active_grid(*G.coarse_dims, device=G.Uc.device)
    phif = active_grid(*G.fine_dims, device=G.Uc.device)
    _call("bsn_solve_fmr_poisson_f64", context(), C.byref(G.s), _ptr(phic), _ptr(phif))
    return phic, phif


# ---------------------------------------------------------------------------
# fast path, device time loop, tile autotuner (no single reference counterpart:
# the reference driver loop test/test_sedov.jl:45-52 run on the device)

PREC = {"f64": 0, "f32": 1, "learned": 2}


def euler3d_step_f32(U, nx, ny, nz, dx, dy, dz, dt, gamma, *, bc="outflow", rho_floor=0.0, P_floor=0.0):
    """euler3d_step! with FP32 stencils/fluxes; FP64 state and RK3 accumulation."""
    _check_state(U, nx, ny, nz)
    _call("bsn_euler3d_step_f32", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz), float(dt),
          float(gamma), BC[bc], float(rho_floor), float(P_floor))


def euler3d_step_learned(U, nx, ny, nz, dx, dy, dz, dt, gamma, *, bc="outflow", rho_floor=0.0, P_floor=0.0):
    """euler3d_step! with the learned WENO weights on smooth stencils (FP32 stencils, FP64 state)."""
    _check_state(U, nx, ny, nz)
    _call("bsn_euler3d_step_learned", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz), float(dt),
          float(gamma), BC[bc], float(rho_floor), float(P_floor))


def run_steps(U, nx, ny, nz, dx, dy, dz, gamma, cfl, *, n_steps, t=0.0, t_end=0.0, bc="outflow", rho_floor=0.0,
              P_floor=0.0, precision="f64"):
    """Up to n_steps CFL-limited RK3 steps on the device; returns (t, steps)."""
    _check_state(U, nx, ny, nz)
    tt = C.c_double(float(t))
    nd = C.c_int(0)
    _call("bsn_run_steps", context(), _ptr(U), nx, ny, nz, float(dx), float(dy), float(dz), float(gamma), float(cfl),
          BC[bc], float(rho_floor), float(P_floor), PREC[precision], int(n_steps), float(t_end), C.byref(tt),
          C.byref(nd))
    return tt.value, nd.value


def tile_variants(precision="f64") -> int:
    return int(load().bsn_tile_variant_count(PREC[precision]))


def set_tma(on=True):
    """Stage the fused kernel's block and halos with TMA tensor copies (the
    default where the grid allows) or with the plain per-thread loader."""
    _call("bsn_ctx_set_tma", context(), int(bool(on)))


def set_stiff_guard(on=True):
    """Uniform-grid FP32 steps: compute faces whose density stencil spans more
    than three decades in FP64 (always on in the driver, FMR and relaxation
    loops)."""
    _call("bsn_ctx_set_stiff_guard", context(), int(bool(on)))


def get_tma() -> bool:
    return bool(load().bsn_ctx_get_tma(context()))


def get_tile_tma(nx, ny, nz, precision="f64"):
    """Whether the tile chosen for this grid is TMA-staged (None: not chosen yet)."""
    r = load().bsn_ctx_get_tile_tma(context(), PREC[precision], nx, ny, nz)
    return None if r < 0 else bool(r)


def set_tile(precision="f64", variant=-1):
    _call("bsn_ctx_set_tile", context(), PREC[precision], int(variant))


def get_tile(nx, ny, nz, precision="f64"):
    """(tx, ty, tz, threads, CTAs per SM) of the tile chosen last for this
    grid; each driver loop keeps its own choice per grid."""
    out = (C.c_int * 5)()
    _call("bsn_ctx_get_tile", context(), PREC[precision], nx, ny, nz, out)
    return tuple(out)


def kernel_time(name: str):
    """(total ms, launches) of kernel `name` since profiling was enabled."""
    tot, cnt = C.c_double(), C.c_longlong()
    _call("bsn_ctx_kernel_stats", context(), name.encode(), C.byref(tot), C.byref(cnt))
    return tot.value, cnt.value


def fp_peak(precision="f64") -> float:
    """Measured FMA throughput in TFLOP/s: "f64", "f32" or "f32x2" (packed)."""
    out = C.c_double()
    _call("bsn_fp_peak", context(), {"f64": 0, "f32": 1, "f32x2": 2}[precision], C.byref(out))
    return out.value


def set_profiling(on: bool):
    _call("bsn_ctx_set_profiling", context(), int(bool(on)))


__all__ += ["euler3d_stage", "add_bh_gravity_source_slab", "add_sink_sources_slab", "gas_force_pairs_slab", "merge_force_pairs",
            "sink_box", "sink_terms_slab", "accrete_from_terms", "euler3d_rhs_f32", "euler3d_step_f32", "euler3d_step_learned", "run_steps", "fmr3d_run_steps", "coupled_run_steps", "diagnostics", "tile_variants", "set_tile", "get_tile", "kernel_time",
            "set_profiling", "fp_peak", "PREC"]
