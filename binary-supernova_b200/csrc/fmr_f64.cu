// fmr_f64.cu -- two-level FMR on the device (src/fmr3d.jl, src/fmr_gravity.jl).
#include "poisson.cuh"

using namespace bsn;

#define BSN_FMR_TODO(name) \
    extern "C" bsn_status name { return set_err(ctx, BSN_ERR_UNSUPPORTED, #name " not built yet"); }

BSN_FMR_TODO(bsn_fmr_prolong_all_f64(bsn_ctx* ctx, const bsn_fmr2*))
BSN_FMR_TODO(bsn_fmr_prolong_fine_ghosts_f64(bsn_ctx* ctx, double*, const double*, const bsn_fmr2*))
BSN_FMR_TODO(bsn_fmr_restrict_f64(bsn_ctx* ctx, double*, const double*, const bsn_fmr2*))
BSN_FMR_TODO(bsn_fmr3d_step_f64(bsn_ctx* ctx, const bsn_fmr2*, double, int, double))
BSN_FMR_TODO(bsn_cfl_dt_fmr3d_f64(bsn_ctx* ctx, const bsn_fmr2*, double, double*))
BSN_FMR_TODO(bsn_restrict_density_to_coarse_f64(bsn_ctx* ctx, const bsn_fmr2*))
BSN_FMR_TODO(bsn_solve_fmr_poisson_f64(bsn_ctx* ctx, const bsn_fmr2*, double*, double*))
