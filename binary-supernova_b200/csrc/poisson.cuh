// poisson.cuh -- isolated-boundary FFT Poisson solver interface (internal).
#pragma once

#include "hydro_f64.cuh"

namespace bsn {

void fft_state_free(bsn_ctx* ctx);
// Allocate and build everything a solve on this grid needs (FFT workspace,
// twiddles, the Green's-function transform) without touching any state, so
// that the solve itself can be captured in a CUDA graph.
bsn_status poisson_prepare(bsn_ctx* ctx, int nx, int ny, int nz, double dx, double dy, double dz);
// The cached FP64 Green's-function transform Khat of the grid (built on first use).
bsn_status poisson_khat64(bsn_ctx* ctx, int nx, int ny, int nz, double dx, double dy, double dz, const double** K);
// FP32-transform counterparts (poisson_f32.cu): FP64 density in, FP64 potential out.
void fft32_state_free(bsn_ctx* ctx);
bsn_status poisson_prepare_f32(bsn_ctx* ctx, int nx, int ny, int nz, double dx, double dy, double dz);
bsn_status poisson_solve_f32(bsn_ctx* ctx, const double* rho, int nx, int ny, int nz, double dx, double dy, double dz,
                             double* phi);
bsn_status poisson_from_state_f32(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy,
                                  double dz, double rho_floor, double* phi);
// Phi = solve_poisson_isolated(rho) for rho on the active grid (nx,ny,nz).
bsn_status poisson_solve(bsn_ctx* ctx, const double* rho, int nx, int ny, int nz, double dx, double dy, double dz,
                         double* phi);
// Same, with rho taken from the state U (density floored at rho_floor when
// rho_floor >= 0, as euler3d_rhs! floors before add_self_gravity_source!).
bsn_status poisson_from_state(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                              double rho_floor, double* phi);
// RK3 step whose every stage solves Poisson on its floored input density.
bsn_status f64_rk3_selfgrav(bsn_ctx* ctx, f64::StageArgs base, double* U, double dt);

}  // namespace bsn
