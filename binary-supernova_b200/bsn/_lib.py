"""ctypes binding of libbsn.so (the C ABI declared in include/bsn.h).

The library is built in-tree (binary-supernova_b200/build_lib.py) and loaded
from this package directory.  There is no fallback: if the shared library is
missing or a CUDA device is absent, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbsn.so")

BSN_OK, BSN_ERR_ARG, BSN_ERR_CUDA, BSN_ERR_TIMEOUT, BSN_ERR_NONFINITE, BSN_ERR_UNSUPPORTED, BSN_ERR_NOMEM = range(7)
_ERRNAMES = {1: "BSN_ERR_ARG", 2: "BSN_ERR_CUDA", 3: "BSN_ERR_TIMEOUT", 4: "BSN_ERR_NONFINITE",
             5: "BSN_ERR_UNSUPPORTED", 6: "BSN_ERR_NOMEM"}


class BSNError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class bsn_bh(C.Structure):
    """Mirror of the reference's mutable BlackHole (src/BinarySupernova.jl:130-137)."""
    _fields_ = [("pos", C.c_double * 3), ("vel", C.c_double * 3), ("mass", C.c_double),
                ("eps", C.c_double), ("c_code", C.c_double), ("r_floor", C.c_double)]

    def __repr__(self):
        return (f"BlackHole(pos={list(self.pos)}, vel={list(self.vel)}, mass={self.mass}, eps={self.eps}, "
                f"c_code={self.c_code}, r_floor={self.r_floor})")


class bsn_fmr2(C.Structure):
    _fields_ = [("Uc", C.c_void_p), ("ncx", C.c_int), ("ncy", C.c_int), ("ncz", C.c_int),
                ("dxc", C.c_double), ("dyc", C.c_double), ("dzc", C.c_double),
                ("Uf", C.c_void_p), ("nfx", C.c_int), ("nfy", C.c_int), ("nfz", C.c_int),
                ("dxf", C.c_double), ("dyf", C.c_double), ("dzf", C.c_double),
                ("ratio", C.c_int),
                ("ci_lo", C.c_int), ("ci_hi", C.c_int), ("cj_lo", C.c_int), ("cj_hi", C.c_int),
                ("ck_lo", C.c_int), ("ck_hi", C.c_int),
                ("gamma", C.c_double), ("bc", C.c_int), ("rho_floor", C.c_double), ("P_floor", C.c_double)]


class bsn_ckpt_meta(C.Structure):
    _fields_ = [("t", C.c_double), ("step", C.c_longlong), ("dt_last", C.c_double), ("t_snap", C.c_double),
                ("t_bh2_sink_on", C.c_double)]


class bsn_grid_meta(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("dz", C.c_double), ("gamma", C.c_double), ("x0", C.c_double), ("y0", C.c_double),
                ("z0", C.c_double), ("rho_floor", C.c_double), ("P_floor", C.c_double)]


class bsn_stage_sources(C.Structure):
    _fields_ = [("bhs", C.POINTER(bsn_bh)), ("nbh", C.c_int), ("nsink", C.c_int), ("f_sink", C.c_double),
                ("torque_free", C.c_int), ("rho_sink_min", C.c_double), ("x0", C.c_double), ("y0", C.c_double),
                ("z0", C.c_double), ("k0", C.c_int), ("phi", C.c_void_p), ("phi_lo", C.c_void_p),
                ("phi_hi", C.c_void_p)]


_V, _I, _D, _P, _LL = C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_longlong
_dp = C.POINTER(C.c_double)
_BH = C.POINTER(bsn_bh)
_FMR = C.POINTER(bsn_fmr2)

# name -> (restype, argtypes); mirrors include/bsn.h
SIGNATURES = {
    "bsn_ctx_create": (_I, [C.POINTER(C.c_void_p), _I, _V]),
    "bsn_ctx_destroy": (_I, [_V]),
    "bsn_ctx_set_stream": (_I, [_V, _V]),
    "bsn_ctx_synchronize": (_I, [_V]),
    "bsn_last_error": (C.c_char_p, [_V]),
    "bsn_version": (C.c_char_p, []),
    "bsn_ctx_launch_count": (_LL, [_V]),
    "bsn_ctx_set_profiling": (_I, [_V, _I]),
    "bsn_ctx_kernel_stats": (_I, [_V, C.c_char_p, _dp, C.POINTER(C.c_longlong)]),
    "bsn_fp_peak": (_I, [_V, _I, _dp]),
    "bsn_fill_ghost_3d_f64": (_I, [_V, _P, _I, _I, _I, _I]),
    "bsn_apply_floors_3d_f64": (_I, [_V, _P, _I, _I, _I, _D, _D, _D]),
    "bsn_euler3d_rhs_f64": (_I, [_V, _P, _P, _P, _P, _P, _I, _I, _I, _D, _D, _D, _D, _I, _D, _D, _I]),
    "bsn_euler3d_step_f64": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _D, _D, _I, _D, _D]),
    "bsn_cfl_dt_3d_f64": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _D, _D, _dp]),
    "bsn_cfl_dt_3d_f64_noalloc": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _D, _D, _dp]),
    "bsn_euler3d_step_f32": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _D, _D, _I, _D, _D]),
    "bsn_run_steps": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _D, _D, _I, _D, _D, _I, _I, _D, _dp,
                           C.POINTER(C.c_int)]),
    "bsn_euler3d_step_learned": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _D, _D, _I, _D, _D]),
    "bsn_learned_param_count": (_I, []),
    "bsn_learned_collect": (_I, [_V, _P, _I, _I, _I, _I, _D, _I, C.c_ulonglong, _P, _P, _LL,
                                 C.POINTER(C.c_longlong)]),
    "bsn_learned_grad": (_I, [_V, _P, _LL, _P, _P, _dp]),
    "bsn_learned_train": (_I, [_V, _P, _LL, _P, _I, _I, C.c_float, C.c_ulonglong, _dp]),
    "bsn_learned_set_params": (_I, [_V, _P, _P]),
    "bsn_learned_eval": (_I, [_V, _P, _LL, _P, _P, _I]),
    "bsn_ctx_set_tma": (_I, [_V, _I]),
    "bsn_ctx_set_stiff_guard": (_I, [_V, _I]),
    "bsn_euler3d_rhs_f32": (_I, [_V, _P, _P, _P, _P, _P, _I, _I, _I, _D, _D, _D, _D, _I, _D, _D, _I]),
    "bsn_ctx_get_tma": (_I, [_V]),
    "bsn_ctx_get_tile_tma": (_I, [_V, _I, _I, _I, _I]),
    "bsn_tile_variant_count": (_I, [_I]),
    "bsn_ctx_set_tile": (_I, [_V, _I, _I]),
    "bsn_ctx_get_tile": (_I, [_V, _I, _I, _I, _I, C.POINTER(C.c_int)]),
    "bsn_add_bh_gravity_source_f64": (_I, [_V, _P, _P, _I, _I, _I, _D, _D, _D, _BH, _I, _D, _D, _D]),
    "bsn_gas_force_on_bh_f64": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _BH, _D, _D, _D, _dp]),
    "bsn_add_sink_sources_f64": (_I, [_V, _P, _P, _I, _I, _I, _D, _D, _D, _BH, _I, _D, _D, _D, _D, _I, _D]),
    "bsn_accrete_f64": (_I, [_V, _BH, _P, _I, _I, _I, _D, _D, _D, _D, _D, _D, _D, _D, _D]),
    "bsn_nbody_step": (_I, [_BH, _I, _D, _dp]),
    "bsn_add_bh_gravity_source_slab_f64": (_I, [_V, _P, _P, _I, _I, _I, _D, _D, _D, _BH, _I, _D, _D, _D, _I]),
    "bsn_add_sink_sources_slab_f64": (_I, [_V, _P, _P, _I, _I, _I, _D, _D, _D, _BH, _I, _D, _D, _D, _D, _I, _D,
                                           _I]),
    "bsn_gas_force_on_bh_slab_f64": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _BH, _D, _D, _D, _I, _dp]),
    "bsn_merge_force_pairs": (_I, [_dp, _I, _dp]),
    "bsn_sink_box": (_I, [_BH, _I, _I, _I, _D, _D, _D, _D, _D, _D, C.POINTER(C.c_int)]),
    "bsn_sink_terms_slab_f64": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _D, _D, _D, _I, _BH, _D, _D, _D,
                                     C.POINTER(C.c_int), _dp, _LL, C.POINTER(C.c_longlong)]),
    "bsn_accrete_from_terms": (_I, [_BH, _dp, _LL]),
    "bsn_euler3d_stage": (_I, [_V, _P, _P, _P, _I, _I, _I, _D, _D, _D, _D, _D, _I, _D, _D, _I,
                               C.POINTER(bsn_stage_sources)]),
    "bsn_save_checkpoint_uniform": (_I, [_V, C.c_char_p, _P, _I, _BH, _I, C.POINTER(bsn_grid_meta),
                                         C.POINTER(bsn_ckpt_meta)]),
    "bsn_save_checkpoint_uniform_async": (_I, [_V, C.c_char_p, _P, _BH, _I, C.POINTER(bsn_grid_meta),
                                               C.POINTER(bsn_ckpt_meta)]),
    "bsn_checkpoint_wait": (_I, [_V]),
    "bsn_load_checkpoint_uniform": (_I, [_V, C.c_char_p, _P, _I, _BH, _I, C.POINTER(C.c_int),
                                         C.POINTER(bsn_grid_meta), C.POINTER(bsn_ckpt_meta)]),
    "bsn_save_checkpoint_fmr": (_I, [_V, C.c_char_p, _FMR, _I, _BH, _I, _D, _LL, _D]),
    "bsn_load_checkpoint_fmr": (_I, [_V, C.c_char_p, _FMR, _I, _BH, _I, C.POINTER(C.c_int), _dp,
                                     C.POINTER(C.c_longlong), _dp]),
    "bsn_write_snapshot": (_I, [_V, C.c_char_p, _P, _I, _I, _I, _I, _D, _D, _D, _D, _D]),
    "bsn_read_snapshot": (_I, [C.c_char_p, _dp, _LL, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                               _dp, _dp, _dp, _dp, _dp]),
    "bsn_trajectory_init": (_I, [C.c_char_p, _I]),
    "bsn_trajectory_append": (_I, [C.c_char_p, _D, _BH, _I]),
    "bsn_trajectory_read": (_I, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _dp, _dp, _dp, _dp,
                                 _LL]),
    "bsn_kepler_init": (_I, [_BH, _dp, _dp, _D, _dp]),
    "bsn_kepler_update": (_I, [_BH, _dp, _D]),
    "bsn_solve_poisson_isolated_f64": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _P]),
    "bsn_poisson_slab_forward_f64": (_I, [_V, _P, _I, _I, _I, _P]),
    "bsn_poisson_slab_zconv_f64": (_I, [_V, _P, _I, _I, _I, _I, _I, _D, _D, _D]),
    "bsn_poisson_slab_inverse_f64": (_I, [_V, _P, _I, _I, _I, _P]),
    "bsn_sg_gradient_f64": (_I, [_V, _P, _P, _P, _I, _I, _I, _D, _D, _D]),
    "bsn_sg_gradient_slab_f64": (_I, [_V, _P, _P, _P, _P, _P, _I, _I, _I, _D, _D, _D]),
    "bsn_add_self_gravity_source_f64": (_I, [_V, _P, _P, _I, _I, _I, _D, _D, _D]),
    "bsn_coupled_step_f64": (_I, [_V, _P, _BH, _I, _D, _D, _I, _I, _I, _D, _D, _D, _D, _D, _D, _D, _D,
                                  _I, _I, _D, _D, _I, _dp]),
    "bsn_coupled_run_steps": (_I, [_V, _P, _BH, _I, _I, _I, _I, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, _I, _I,
                                   _D, _D, _I, _I, _I, _D, _dp, C.POINTER(C.c_int), _P, _I]),
    "bsn_diagnostics_f64": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _D, _D, _D, _BH, _I, _D, _dp]),
    "bsn_rotating_frame_source_f64": (_I, [_V, _P, _P, _I, _I, _I, _D, _D, _D, _D, _D, _D, _D]),
    "bsn_relax_damping_source_f64": (_I, [_V, _P, _P, _I, _I, _I, _D, _D, _D, _D, _D, _D, _D, _D]),
    "bsn_relax_ic": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _D, _BH, _I, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D,
                          _I, _I, _I, _dp, C.POINTER(C.c_int), _dp]),
    "bsn_coupled_nested_run_steps": (_I, [_V, _FMR, _I, _BH, _I, _D, _D, _D, _D, _D, _D, _I, _I, _D, _D, _I, _I,
                                          _I, _D, _dp, C.POINTER(C.c_int), _P, _I]),
    "bsn_fmr_prolong_all_f64": (_I, [_V, _FMR]),
    "bsn_fmr_prolong_fine_ghosts_f64": (_I, [_V, _P, _P, _FMR]),
    "bsn_fmr_restrict_f64": (_I, [_V, _P, _P, _FMR]),
    "bsn_fmr3d_step_f64": (_I, [_V, _FMR, _D, _I, _D]),
    "bsn_cfl_dt_fmr3d_f64": (_I, [_V, _FMR, _D, _dp]),
    "bsn_restrict_density_to_coarse_f64": (_I, [_V, _FMR]),
    "bsn_solve_fmr_poisson_f64": (_I, [_V, _FMR, _P, _P]),
    "bsn_prolong_scalar_trilinear_f64": (_I, [_V, _FMR, _P, _P]),
    "bsn_solve_poisson_isolated_f32": (_I, [_V, _P, _I, _I, _I, _D, _D, _D, _P]),
    "bsn_fmr3d_run_steps": (_I, [_V, _FMR, _D, _I, _I, _D, _I, _D, _dp, C.POINTER(C.c_int)]),
    "bsn_fmr_nested_step_f64": (_I, [_V, _FMR, _I, _D, _I, _D]),
    "bsn_cfl_dt_fmr_nested_f64": (_I, [_V, _FMR, _I, _D, _dp]),
    "bsn_fmr_nested_run_steps": (_I, [_V, _FMR, _I, _D, _I, _I, _D, _I, _D, _dp, C.POINTER(C.c_int)]),
}

_lib = None
_lock = threading.Lock()


def load():
    """Load libbsn.so and declare every exported entry point."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"libbsn.so not found at {LIB_PATH}: build it with "
                                   "`python binary-supernova_b200/build_lib.py` (no CPU fallback exists)")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def exported_symbols():
    return sorted(SIGNATURES)
