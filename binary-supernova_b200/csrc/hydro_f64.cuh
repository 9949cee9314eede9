// hydro_f64.cuh -- internal interface of the FP64 uniform-grid path, shared by
// the coupled step, self-gravity and FMR drivers.
#pragma once

#include <cmath>
#include <cstring>
#include <algorithm>

#include "stage_f64.cuh"

namespace bsn {

bsn_status check_dims(bsn_ctx* ctx, int nx, int ny, int nz);
bsn_status f64_fill_ghosts(bsn_ctx* ctx, double* U, int nx, int ny, int nz, int bc);
// Cells of a half-open box [lo, hi) of active indices (lo = hi: none).
struct LedBox {
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    __host__ __device__ bool has(int a, int b, int c) const {
        return a >= lo[0] && a < hi[0] && b >= lo[1] && b < hi[1] && c >= lo[2] && c < hi[2];
    }
};
// apply_floors_3d! on the active cells; with led, the floors' change of the
// mass outside `skip` (rho dV, dV the cell volume) is added to *led.
bsn_status f64_floors(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double rho_floor, double P_floor, double gamma,
                      const int* done_dev = nullptr, double* led = nullptr, LedBox skip = LedBox{}, double dV = 0.0);
// Fold one RK3 step's per-stage mass-ledger sums raw[3][LED_TERMS] into the
// cumulative totals tot[LEDT_COUNT] with the step's dt (hydro_f64.cu).
bsn_status f64_ledger_fold(bsn_ctx* ctx, double* raw, double* tot, const double* dt_dev, const int* done_dev);
bsn_status f64_ghost_combine(bsn_ctx* ctx, double* U, const double* S, const double* Gh, int nx, int ny, int nz,
                             int bc, double dt, const double* dt_dev = nullptr, const int* done_dev = nullptr);
void stage_args_init(f64::StageArgs& A, int nx, int ny, int nz, double dx, double dy, double dz, double gamma, int bc,
                     double rho_floor, double P_floor);
void set_stage(f64::StageArgs& A, int stage, double dt);
bsn_status f64_launch_stage(bsn_ctx* ctx, const f64::StageArgs& A);
bsn_status f64_rk3(bsn_ctx* ctx, f64::StageArgs base, double* U, double dt, const double* phi_per_stage[3],
                   unsigned long long* cfl_max, unsigned int* cfl_nan);
bsn_status f64_cfl_dt(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                      double gamma, double cfl, double* dt_out);
bsn_status f64_cfl_fold(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                        double gamma, unsigned long long* smax, unsigned int* nanflag);
bsn_status cfl_from_device(bsn_ctx* ctx, const unsigned long long* red, double cfl, double* dt_out);
// Replay a one-step graph up to n_steps times on ctx->stream.  With
// until_done, replays go in chunks and stop once the device flag *done_dev
// is set (each chunk's flag is read back behind it; the host waits for the
// previous chunk's flag only after queueing the next).  ev: two events,
// hflag: two pinned ints.
bsn_status graph_replay(bsn_ctx* ctx, cudaGraphExec_t exec, int kernels, int n_steps, bool until_done,
                        const int* done_dev, cudaEvent_t ev[2], volatile int* hflag);

// r_sink / t_sink of src/BinarySupernova.jl:159-171 (host FP64).
inline double bh_r_sink(const bsn_bh& b) {
    double v = 6.0 * b.mass / (b.c_code * b.c_code);
    return jmax(v, b.r_floor);
}
inline double bh_t_sink(const bsn_bh& b, double f_sink) {
    double rs = bh_r_sink(b);
    double v_ff = std::sqrt(2.0 * b.mass / rs);
    return f_sink * rs / v_ff;
}

}  // namespace bsn
