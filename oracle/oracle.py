"""ctypes front end for the CPU FP64 oracle (liboracle: oracle/bsn_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py.  The product path (libbsn + the bsn package)
never imports this module.

Arrays follow the reference's Julia layout: numpy Fortran-ordered float64 of
shape (5, nx+6, ny+6, nz+6), so ``U[q, i, j, k]`` (0-based) is the reference's
``U[q+1, i+1, j+1, k+1]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

NG = 3
_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "libbsn_oracle.so")

_dp = C.POINTER(C.c_double)


class OrcBH(C.Structure):
    """Mirror of the reference BlackHole (src/BinarySupernova.jl:130-137)."""
    _fields_ = [("pos", C.c_double * 3), ("vel", C.c_double * 3), ("mass", C.c_double),
                ("eps", C.c_double), ("c_code", C.c_double), ("r_floor", C.c_double)]


class OrcFMR(C.Structure):
    _fields_ = [("Uc", _dp), ("ncx", C.c_int), ("ncy", C.c_int), ("ncz", C.c_int),
                ("dxc", C.c_double), ("dyc", C.c_double), ("dzc", C.c_double),
                ("Uf", _dp), ("nfx", C.c_int), ("nfy", C.c_int), ("nfz", C.c_int),
                ("dxf", C.c_double), ("dyf", C.c_double), ("dzf", C.c_double),
                ("ratio", C.c_int),
                ("ci_lo", C.c_int), ("ci_hi", C.c_int), ("cj_lo", C.c_int), ("cj_hi", C.c_int),
                ("ck_lo", C.c_int), ("ck_hi", C.c_int),
                ("gamma", C.c_double), ("bc", C.c_int),
                ("rho_floor", C.c_double), ("P_floor", C.c_double)]


def build() -> str:
    """Compile liboracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    d, i, P, V = C.c_double, C.c_int, _dp, None
    sig = {
        "orc_weno5_left": (d, [d] * 5), "orc_weno5_right": (d, [d] * 5),
        "orc_wenoz_weights": (V, [d] * 6 + [P]),
        "orc_hllc_flux": (V, [i, P, P, d, P]),
        "orc_set_threads": (V, [i]),
        "orc_fill_ghost_outflow": (V, [P, i, i, i]), "orc_fill_ghost_periodic": (V, [P, i, i, i]),
        "orc_apply_floors": (V, [P, i, i, i, d, d, d]),
        "orc_weno_fluxes": (V, [i, P, P, i, i, i, d]),
        "orc_flux_divergence": (V, [P, P, P, P, i, i, i, d, d, d]),
        "orc_cfl_dt_3d": (d, [P, i, i, i, d, d, d, d, d]),
        "orc_euler3d_rhs": (V, [P, P, P, P, P, i, i, i, d, d, d, d, i, d, d, i]),
        "orc_euler3d_step": (V, [P, i, i, i, d, d, d, d, d, i, d, d]),
        "orc_sedov_ic_3d": (V, [P, i, i, i, d, d, d, d, d, d, d, d, d, d, d]),
        "orc_r_sink": (d, [C.POINTER(OrcBH)]), "orc_t_sink": (d, [C.POINTER(OrcBH), d]),
        "orc_add_bh_gravity_source": (V, [P, P, i, i, i, d, d, d, C.POINTER(OrcBH), i, d, d, d]),
        "orc_gas_force_on_bh": (V, [P, i, i, i, d, d, d, C.POINTER(OrcBH), d, d, d, P]),
        "orc_add_sink_sources": (V, [P, P, i, i, i, d, d, d, C.POINTER(OrcBH), i, d, d, d, d, i, d]),
        "orc_accrete": (V, [C.POINTER(OrcBH), P, i, i, i, d, d, d, d, d, d, d, d, d]),
        "orc_add_bh_gravity_source_slab": (V, [P, P, i, i, i, d, d, d, C.POINTER(OrcBH), i, d, d, d, i]),
        "orc_gas_force_on_bh_slab": (V, [P, i, i, i, d, d, d, C.POINTER(OrcBH), d, d, d, i, P]),
        "orc_add_sink_sources_slab": (V, [P, P, i, i, i, d, d, d, C.POINTER(OrcBH), i, d, d, d, d, i, d, i]),
        "orc_sink_terms_slab": (C.c_long, [P, i, i, i, d, d, d, d, d, d, i, C.POINTER(OrcBH), d, d,
                                           i, i, i, i, i, i, P]),
        "orc_nbody_step": (V, [C.POINTER(OrcBH), i, d, P]),
        "orc_kepler_init": (i, [C.POINTER(OrcBH), P, P, d, P]),
        "orc_kepler_update": (V, [C.POINTER(OrcBH), P, d]),
        "orc_fft3d": (V, [P, P, i, i, i, i]),
        "orc_solve_poisson_isolated": (V, [P, i, i, i, d, d, d, P]),
        "orc_sg_gradient": (V, [P, P, P, i, i, i, d, d, d]),
        "orc_add_self_gravity_source": (V, [P, P, i, i, i, d, d, d]),
        "orc_coupled_step": (V, [P, P, P, P, P, P, C.POINTER(OrcBH), i, d, d, i, i, i, d, d, d, d,
                                 d, d, d, d, i, i, d, d, i, P]),
        "orc_lag5_weights": (V, [i, P]),
        "orc_prolong_all": (V, [C.POINTER(OrcFMR)]),
        "orc_prolong_fine_ghosts": (V, [P, P, C.POINTER(OrcFMR)]),
        "orc_restrict": (V, [P, P, C.POINTER(OrcFMR)]),
        "orc_fmr3d_step": (V, [C.POINTER(OrcFMR), d, i, d]),
        "orc_cfl_dt_fmr3d": (d, [C.POINTER(OrcFMR), d]),
        "orc_fmrN_step": (V, [C.POINTER(OrcFMR), i, d, i, d]),
        "orc_cfl_dt_fmrN": (d, [C.POINTER(OrcFMR), i, d]),
        "orc_gas_force_fmrN": (V, [C.POINTER(OrcFMR), i, C.POINTER(OrcBH), d, d, d, P]),
        "orc_rotating_frame_source": (V, [P, P, i, i, i, d, d, d, d, d, d, d]),
        "orc_relax_damping_source": (V, [P, P, i, i, i, d, d, d, d, d, d, d, d]),
        "orc_relax_ic": (V, [P, i, i, i, d, d, d, d, C.POINTER(OrcBH), i, d, d, d, d, d, d, d, d, d, d, i, i, P]),
        "orc_coupled_fmrN_step": (V, [C.POINTER(OrcFMR), i, C.POINTER(OrcBH), i, d, d, d, d, d, d, i, i, d, d, i,
                                      P]),
        "orc_restrict_density_to_coarse": (V, [C.POINTER(OrcFMR)]),
        "orc_prolong_scalar_trilinear": (V, [P, P, C.POINTER(OrcFMR)]),
        "orc_solve_fmr_poisson": (V, [C.POINTER(OrcFMR), P, P]),
        "orc_lane_emden": (i, [d, d, P, P, P, i]),
        "orc_polytrope_ic_3d": (V, [P, i, i, i, d, d, d, d, d, d, d, d, d, d, d, d, d, d, d, P]),
        "orc_thermal_bomb": (d, [P, i, i, i] + [d] * 13),
        "orc_diagnostics": (V, [P, i, i, i, d, d, d, d, d, d, C.POINTER(OrcBH), i, d, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim <= 1), "need F-ordered float64"
    return a.ctypes.data_as(_dp)


# --------------------------------------------------------------------------
# array helpers

def state(nx: int, ny: int, nz: int) -> np.ndarray:
    return np.zeros((5, nx + 2 * NG, ny + 2 * NG, nz + 2 * NG), dtype=np.float64, order="F")


def flux_arrays(nx: int, ny: int, nz: int):
    X, Y, Z = nx + 2 * NG, ny + 2 * NG, nz + 2 * NG
    return (np.zeros((5, X + 1, Y, Z), order="F"), np.zeros((5, X, Y + 1, Z), order="F"),
            np.zeros((5, X, Y, Z + 1), order="F"))


def dims(U: np.ndarray):
    return U.shape[1] - 2 * NG, U.shape[2] - 2 * NG, U.shape[3] - 2 * NG


BC = {"outflow": 0, "periodic": 1}


def set_threads(n: int):
    lib().orc_set_threads(int(n))


# --------------------------------------------------------------------------
# reference entry points (same names and argument meaning as the Julia)

def weno5_left(*v):
    return lib().orc_weno5_left(*map(float, v))


def weno5_right(*v):
    return lib().orc_weno5_right(*map(float, v))


def hllc_flux(direction: int, L, R, gamma: float):
    Ld = (C.c_double * 5)(*L)
    Rd = (C.c_double * 5)(*R)
    out = (C.c_double * 5)()
    lib().orc_hllc_flux(direction, Ld, Rd, gamma, out)
    return tuple(out)


def fill_ghost_3d_outflow(U):
    lib().orc_fill_ghost_outflow(_p(U), *dims(U))


def fill_ghost_3d_periodic(U):
    lib().orc_fill_ghost_periodic(_p(U), *dims(U))


def apply_floors_3d(U, rho_floor, P_floor, gamma):
    lib().orc_apply_floors(_p(U), *dims(U), rho_floor, P_floor, gamma)


def euler3d_rhs(dU, Fx, Fy, Fz, U, dx, dy, dz, gamma, bc="outflow", rho_floor=0.0, P_floor=0.0,
                fill_ghosts=True):
    lib().orc_euler3d_rhs(_p(dU), _p(Fx), _p(Fy), _p(Fz), _p(U), *dims(U), dx, dy, dz, gamma,
                          BC[bc], rho_floor, P_floor, int(fill_ghosts))


def euler3d_step(U, dx, dy, dz, dt, gamma, bc="outflow", rho_floor=0.0, P_floor=0.0):
    lib().orc_euler3d_step(_p(U), *dims(U), dx, dy, dz, dt, gamma, BC[bc], rho_floor, P_floor)


def cfl_dt_3d(U, dx, dy, dz, gamma, cfl):
    return lib().orc_cfl_dt_3d(_p(U), *dims(U), dx, dy, dz, gamma, cfl)


_flops_lib = None
FLOP_KINDS = ("add", "mul", "div", "sqrt", "cmp")


def count_step_flops(U, dx, dy, dz, dt, gamma, bc="outflow", rho_floor=0.0, P_floor=0.0) -> dict:
    """euler3d_step! on U (in place, the oracle's arithmetic) through the
    counting build (oracle/flops.cpp); returns the operations it took:
    add (+ and -), mul, div, sqrt, cmp, one each, and their total."""
    global _flops_lib
    if _flops_lib is None:
        path = os.path.join(_HERE, "build", "libbsn_oracle_flops.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        d, i = C.c_double, C.c_int
        L.orc_count_step.restype = None
        L.orc_count_step.argtypes = [_dp, i, i, i, d, d, d, d, d, i, d, d, C.c_ulonglong * 5]
        _flops_lib = L
    out = (C.c_ulonglong * 5)()
    _flops_lib.orc_count_step(_p(U), *dims(U), dx, dy, dz, dt, gamma, BC[bc], rho_floor, P_floor, out)
    r = dict(zip(FLOP_KINDS, (int(v) for v in out)))
    r["total"] = sum(out)
    return r


def sedov_ic_3d(U, dx, dy, dz, gamma, E_blast=1.0, r_inject=None, rho_bg=1.0, P_floor=1e-5,
                x_offset=0.0, y_offset=0.0, z_offset=0.0):
    lib().orc_sedov_ic_3d(_p(U), *dims(U), dx, dy, dz, gamma, E_blast,
                          -1.0 if r_inject is None else float(r_inject), rho_bg, P_floor,
                          x_offset, y_offset, z_offset)


def make_bh(pos, vel, mass, eps, c_code, r_floor) -> OrcBH:
    return OrcBH((C.c_double * 3)(*pos), (C.c_double * 3)(*vel), mass, eps, c_code, r_floor)


def bh_array(bhs):
    arr = (OrcBH * max(1, len(bhs)))()
    for t, b in enumerate(bhs):
        arr[t] = b
    return arr


def r_sink(bh: OrcBH):
    return lib().orc_r_sink(C.byref(bh))


def t_sink(bh: OrcBH, f_sink=1.0):
    return lib().orc_t_sink(C.byref(bh), f_sink)


def add_bh_gravity_source(dU, U, dx, dy, dz, bhs, x0, y0, z0):
    arr = bh_array(bhs)
    lib().orc_add_bh_gravity_source(_p(dU), _p(U), *dims(U), dx, dy, dz, arr, len(bhs), x0, y0, z0)


def gas_force_on_bh(U, dx, dy, dz, bh, x0, y0, z0):
    out = (C.c_double * 3)()
    lib().orc_gas_force_on_bh(_p(U), *dims(U), dx, dy, dz, C.byref(bh), x0, y0, z0, out)
    return np.array(out[:])


def add_sink_sources(dU, U, dx, dy, dz, bhs, x0, y0, z0, f_sink=1.0, torque_free=True, rho_sink_min=0.0):
    arr = bh_array(bhs)
    lib().orc_add_sink_sources(_p(dU), _p(U), *dims(U), dx, dy, dz, arr, len(bhs), x0, y0, z0,
                               f_sink, int(torque_free), rho_sink_min)


def accrete(bh: OrcBH, U, dx, dy, dz, x0, y0, z0, dt, f_sink=1.0, rho_sink_min=0.0):
    lib().orc_accrete(C.byref(bh), _p(U), *dims(U), dx, dy, dz, x0, y0, z0, dt, f_sink, rho_sink_min)


def add_bh_gravity_source_slab(dU, U, dx, dy, dz, bhs, x0, y0, z0, kofs):
    """add_bh_gravity_source! on a z-slab whose first active plane is global plane kofs."""
    arr = bh_array(bhs)
    lib().orc_add_bh_gravity_source_slab(_p(dU), _p(U), *dims(U), dx, dy, dz, arr, len(bhs), x0, y0, z0, kofs)


def gas_force_on_bh_slab(U, dx, dy, dz, bh, x0, y0, z0, kofs):
    out = (C.c_double * 3)()
    lib().orc_gas_force_on_bh_slab(_p(U), *dims(U), dx, dy, dz, C.byref(bh), x0, y0, z0, kofs, out)
    return np.array(out[:])


def add_sink_sources_slab(dU, U, dx, dy, dz, bhs, x0, y0, z0, kofs, f_sink=1.0, torque_free=True, rho_sink_min=0.0):
    arr = bh_array(bhs)
    lib().orc_add_sink_sources_slab(_p(dU), _p(U), *dims(U), dx, dy, dz, arr, len(bhs), x0, y0, z0,
                                    f_sink, int(torque_free), rho_sink_min, kofs)


def sink_terms_slab(U, dx, dy, dz, x0, y0, z0, kofs, bh, rate, rho_sink_min, box):
    """accrete!'s per-cell terms over this slab's part of the global box (k, j, i order), (n, 4)."""
    ilo, ihi, jlo, jhi, klo, khi = box
    nz = dims(U)[2]
    n = max(0, ihi - ilo + 1) * max(0, jhi - jlo + 1) * max(0, min(khi, kofs + nz - 1) - max(klo, kofs) + 1)
    out = np.zeros((max(n, 1), 4))
    m = lib().orc_sink_terms_slab(_p(U), *dims(U), dx, dy, dz, x0, y0, z0, kofs, C.byref(bh), rate, rho_sink_min,
                                  ilo, ihi, jlo, jhi, klo, khi, out.ctypes.data_as(_dp))
    assert m == n
    return out[:n]


def nbody_step(bhs_arr, nbh, dt, F_gas: np.ndarray):
    F = np.ascontiguousarray(F_gas, dtype=np.float64).reshape(-1)
    lib().orc_nbody_step(bhs_arr, nbh, dt, F.ctypes.data_as(_dp))


def kepler_init(bhs_arr, com=(0.0, 0.0, 0.0), nhat=None, Omega=None):
    st = np.zeros(13)
    c = np.array(com, dtype=np.float64)
    nh = None if nhat is None else np.array(nhat, dtype=np.float64)
    rc = lib().orc_kepler_init(bhs_arr, c.ctypes.data_as(_dp),
                               None if nh is None else nh.ctypes.data_as(_dp),
                               -1.0 if Omega is None else float(Omega), st.ctypes.data_as(_dp))
    if rc != 0:
        raise ValueError(f"KeplerOrbit construction failed ({rc})")
    return st


def kepler_update(bhs_arr, st, t):
    lib().orc_kepler_update(bhs_arr, st.ctypes.data_as(_dp), t)


def solve_poisson_isolated(rho: np.ndarray, dx, dy, dz):
    rho = np.asfortranarray(rho, dtype=np.float64)
    phi = np.zeros_like(rho, order="F")
    lib().orc_solve_poisson_isolated(_p(rho), *rho.shape, dx, dy, dz, _p(phi))
    return phi


def sg_gradient(dU, U, phi, dx, dy, dz):
    lib().orc_sg_gradient(_p(dU), _p(U), _p(np.asfortranarray(phi)), *dims(U), dx, dy, dz)


def add_self_gravity_source(dU, U, dx, dy, dz):
    lib().orc_add_self_gravity_source(_p(dU), _p(U), *dims(U), dx, dy, dz)


def rotating_frame_source(dU, U, dx, dy, dz, x0, y0, z0, Omega):
    lib().orc_rotating_frame_source(_p(dU), _p(U), *dims(U), dx, dy, dz, x0, y0, z0, Omega)


def relax_damping_source(dU, U, dx, dy, dz, x0, y0, z0, t_damp, Omega=0.0):
    lib().orc_relax_damping_source(_p(dU), _p(U), *dims(U), dx, dy, dz, x0, y0, z0, t_damp, Omega)


def relax_ic(U, dx, dy, dz, gamma, bhs=(), x0=0.0, y0=0.0, z0=0.0, t_damp=0.1, t_max=2.0, cfl=0.4,
             rho_floor=1e-10, P_floor=1e-10, KE_tol=0.01, Omega=0.0, self_gravity=False, max_steps=1000000):
    """relax_ic! (src/relax_ic.jl:200-330); returns (t, n_steps, KE_ratio)."""
    arr = bh_array(list(bhs))
    out = np.zeros(3)
    lib().orc_relax_ic(_p(U), *dims(U), dx, dy, dz, gamma, arr, len(bhs), x0, y0, z0, t_damp, t_max, cfl,
                       rho_floor, P_floor, KE_tol, Omega, int(self_gravity), int(max_steps), out.ctypes.data_as(_dp))
    return float(out[0]), int(out[1]), float(out[2])


def coupled_step(U, bhs_arr, nbh, dt, t, dx, x0, y0, z0, gamma, f_sink, rho_floor, P_floor,
                 torque_free, self_gravity, t_bh2_sink_on, rho_sink_min, evolve_orbit=True):
    nx, ny, nz = dims(U)
    Un = np.zeros_like(U, order="F")
    dU = np.zeros_like(U, order="F")
    Fx, Fy, Fz = flux_arrays(nx, ny, nz)
    Fg = np.zeros(3 * max(nbh, 1))
    lib().orc_coupled_step(_p(U), _p(Un), _p(dU), _p(Fx), _p(Fy), _p(Fz), bhs_arr, nbh, dt, t,
                           nx, ny, nz, dx, x0, y0, z0, gamma, f_sink, rho_floor, P_floor,
                           int(torque_free), int(self_gravity), t_bh2_sink_on, rho_sink_min,
                           int(evolve_orbit), Fg.ctypes.data_as(_dp))
    return Fg[: 3 * nbh].reshape(nbh, 3)


# --------------------------------------------------------------------------
# FMR

class FMRGrid:
    """Two-level FMR grid (src/fmr3d.jl:109-151) holding numpy level arrays."""

    def __init__(self, Uc, dxc, ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi, ratio, gamma,
                 bc="outflow", rho_floor=0.0, P_floor=0.0, dyc=None, dzc=None, init=True):
        ncx, ncy, ncz = dims(Uc)
        dyc = dxc if dyc is None else dyc
        dzc = dxc if dzc is None else dzc
        nfx, nfy, nfz = ((ci_hi - ci_lo + 1) * ratio, (cj_hi - cj_lo + 1) * ratio,
                         (ck_hi - ck_lo + 1) * ratio)
        self.Uc = Uc
        self.Uf = state(nfx, nfy, nfz)
        self.s = OrcFMR(_p(self.Uc), ncx, ncy, ncz, dxc, dyc, dzc,
                        _p(self.Uf), nfx, nfy, nfz, dxc / ratio, dyc / ratio, dzc / ratio,
                        ratio, ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi, gamma, BC[bc],
                        rho_floor, P_floor)
        if init:
            lib().orc_prolong_all(C.byref(self.s))

    def prolong_fine_ghosts(self, Uc_src=None):
        src = self.Uc if Uc_src is None else Uc_src
        lib().orc_prolong_fine_ghosts(_p(self.Uf), _p(src), C.byref(self.s))

    def restrict(self):
        lib().orc_restrict(_p(self.Uc), _p(self.Uf), C.byref(self.s))

    def step(self, dt_c, self_gravity=False, G_grav=1.0):
        lib().orc_fmr3d_step(C.byref(self.s), dt_c, int(self_gravity), G_grav)

    def cfl_dt(self, cfl):
        return lib().orc_cfl_dt_fmr3d(C.byref(self.s), cfl)

    def restrict_density_to_coarse(self):
        lib().orc_restrict_density_to_coarse(C.byref(self.s))

    def prolong_scalar_trilinear(self, phic):
        s = self.s
        phif = np.zeros((s.nfx, s.nfy, s.nfz), order="F")
        lib().orc_prolong_scalar_trilinear(_p(phif), _p(np.asfortranarray(phic)), C.byref(s))
        return phif

    def solve_poisson(self):
        s = self.s
        phic = np.zeros((s.ncx, s.ncy, s.ncz), order="F")
        phif = np.zeros((s.nfx, s.nfy, s.nfz), order="F")
        lib().orc_solve_fmr_poisson(C.byref(s), _p(phic), _p(phif))
        return phic, phif


class FMRHierarchy:
    """N nested levels: a chain of FMRGrid pairs where pair k's fine level is
    pair k+1's coarse level.  levels[0] is the base grid; each entry of
    `boxes` is (ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi, ratio) in the
    interior indices of the level above it."""

    def __init__(self, U0, dx0, boxes, gamma, bc="outflow", rho_floor=0.0, P_floor=0.0):
        self.pairs = []
        Uc, dxc = U0, dx0
        for (a, b, c, d_, e, f, r) in boxes:
            g = FMRGrid(Uc, dxc, a, b, c, d_, e, f, r, gamma, bc=bc, rho_floor=rho_floor,
                        P_floor=P_floor)
            self.pairs.append(g)
            Uc, dxc = g.Uf, dxc / r
        self.levels = [U0] + [g.Uf for g in self.pairs]
        self._arr = (OrcFMR * len(self.pairs))(*[g.s for g in self.pairs])

    def step(self, dt0, self_gravity=False, G_grav=1.0):
        lib().orc_fmrN_step(self._arr, len(self.pairs), dt0, int(self_gravity), G_grav)

    def cfl_dt(self, cfl):
        return lib().orc_cfl_dt_fmrN(self._arr, len(self.pairs), cfl)

    def gas_force(self, bh, x0, y0, z0):
        out = np.zeros(3)
        lib().orc_gas_force_fmrN(self._arr, len(self.pairs), C.byref(bh), x0, y0, z0, out.ctypes.data_as(_dp))
        return out

    def coupled_step(self, bhs_arr, nbh, dt0, t, x0, y0, z0, f_sink, torque_free, self_gravity, t_bh2_sink_on,
                     rho_sink_min, evolve_orbit=True):
        """coupled_step! on the nested levels (composite gas force, orbit,
        nested step with sources on every level, accretion on the finest)."""
        Fg = np.zeros(3 * max(nbh, 1))
        lib().orc_coupled_fmrN_step(self._arr, len(self.pairs), bhs_arr, nbh, dt0, t, x0, y0, z0, f_sink,
                                    int(torque_free), int(self_gravity), t_bh2_sink_on, rho_sink_min,
                                    int(evolve_orbit), Fg.ctypes.data_as(_dp))
        return Fg[: 3 * nbh].reshape(nbh, 3)


def lag5_weights(ratio):
    w = np.zeros((ratio, 5), order="F")
    lib().orc_lag5_weights(ratio, _p(w))
    return w


# --------------------------------------------------------------------------
# input generators

def polytrope_ic_3d(U, dx, dy, dz, gamma, M_star, R_star, x0=0.0, y0=0.0, z0=0.0,
                    x_center=0.0, y_center=0.0, z_center=0.0, rho_floor=1e-10, P_floor=1e-8):
    out = np.zeros(4)
    lib().orc_polytrope_ic_3d(_p(U), *dims(U), dx, dy, dz, gamma, M_star, R_star, 0.0, x0, y0, z0,
                              x_center, y_center, z_center, rho_floor, P_floor, out.ctypes.data_as(_dp))
    return tuple(out)


def thermal_bomb(U, dx, dy, dz, E_SN, r_bomb, r_bomb_inner=0.0, x0=0.0, y0=0.0, z0=0.0,
                 x_center=0.0, y_center=0.0, z_center=0.0, bipolar_theta_deg=180.0):
    return lib().orc_thermal_bomb(_p(U), *dims(U), dx, dy, dz, E_SN, r_bomb, r_bomb_inner, x0, y0, z0,
                                  x_center, y_center, z_center, bipolar_theta_deg)


def sod_ic_3d(direction: str, n_normal=128, n_trans=4, gamma=1.4):
    """test/test_sod3d.jl:146-171 initial state."""
    nx, ny, nz = {"x": (n_normal, n_trans, n_trans), "y": (n_trans, n_normal, n_trans),
                  "z": (n_trans, n_trans, n_normal)}[direction]
    dx, dy, dz = 1.0 / nx, 1.0 / ny, 1.0 / nz
    U = state(nx, ny, nz)
    ax = "xyz".index(direction)
    n = (nx, ny, nz)[ax]
    d = (dx, dy, dz)[ax]
    coord = (np.arange(1, n + 1) - 0.5) * d - 0.5
    left = coord < 0.0
    rho = np.where(left, 1.0, 0.125)
    pr = np.where(left, 1.0, 0.1)
    E = pr / (gamma - 1) + 0.5 * rho * 0.0 ** 2
    shape = [1, 1, 1]
    shape[ax] = n
    act = (slice(NG, NG + nx), slice(NG, NG + ny), slice(NG, NG + nz))
    U[(0,) + act] = np.broadcast_to(rho.reshape(shape), (nx, ny, nz))
    U[(4,) + act] = np.broadcast_to(E.reshape(shape), (nx, ny, nz))
    return U, (nx, ny, nz), (dx, dy, dz)


def diagnostics(U, dx, dy, dz, x0, y0, z0, bhs, gamma):
    """src/diagnostics.jl: (E_gas, KE_gas, Px, Py, Pz, Lx, Ly, Lz, M_bound, M_gas)."""
    out = np.zeros(10)
    arr = bh_array(bhs)
    lib().orc_diagnostics(_p(U), *dims(U), dx, dy, dz, x0, y0, z0, arr, len(bhs), gamma,
                          out.ctypes.data_as(_dp))
    return out
