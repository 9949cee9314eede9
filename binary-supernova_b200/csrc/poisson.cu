// poisson.cu -- isolated FFT Poisson solve (src/self_gravity.jl:35-76).
#include "poisson.cuh"

namespace bsn {

void fft_state_free(bsn_ctx*) {}

bsn_status poisson_solve(bsn_ctx* ctx, const double*, int, int, int, double, double, double, double*) {
    return set_err(ctx, BSN_ERR_UNSUPPORTED, "Poisson solver not built yet");
}
bsn_status poisson_from_state(bsn_ctx* ctx, const double*, int, int, int, double, double, double, double, double*) {
    return set_err(ctx, BSN_ERR_UNSUPPORTED, "Poisson solver not built yet");
}
bsn_status f64_rk3_selfgrav(bsn_ctx* ctx, f64::StageArgs, double*, double) {
    return set_err(ctx, BSN_ERR_UNSUPPORTED, "Poisson solver not built yet");
}

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_solve_poisson_isolated_f64(bsn_ctx* ctx, const double* rho, int nx, int ny, int nz, double dx,
                                                     double dy, double dz, double* phi) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    return poisson_solve(ctx, rho, nx, ny, nz, dx, dy, dz, phi);
}
