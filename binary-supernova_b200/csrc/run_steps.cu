// run_steps.cu -- device-resident time stepping with one CUDA graph per step.
//
// The reference's driver loop (`dt = cfl_dt_3d(U); dt = min(dt, t_end - t);
// euler3d_step!(...); t += dt`, test/test_sedov.jl:45-52) costs a host round
// trip per step for dt.  Here dt, t and the CFL maximum live on the device:
// the stage-3 kernel folds the next step's CFL speed while it writes the new
// state, a one-thread kernel turns it into dt (and stops the loop once t
// reaches t_end: later launches return at once), and the whole step -- dt,
// three fused stages, final ghost values, t += dt -- is captured once into a
// CUDA graph and replayed.  The arithmetic is that of the per-step entry
// points, so the FP64 path stays bit-identical to the reference.
#include "hydro_f64.cuh"
#include "stage_launch.cuh"

namespace bsn {
namespace run {

struct Dev {
    double dt, t;
    unsigned long long smax;
    unsigned int nanflag;
    int done;
    int steps;
    int pad;
};

__global__ void init_kernel(Dev* r, double t) {
    r->dt = 0.0; r->t = t; r->smax = 0ull; r->nanflag = 0u; r->done = 0; r->steps = 0;
}

// dt = cfl / max speed (Inf when the max is 0 or NaN, as the reference);
// with t_end > 0: stop when t >= t_end, else dt = min(dt, t_end - t).
__global__ void dt_kernel(Dev* r, double cfl, double t_end) {
    if (r->done) return;
    double smax = __longlong_as_double((long long)r->smax);
    double dt = r->nanflag ? INFINITY : (smax > 0.0 ? cfl / smax : INFINITY);
    if (t_end > 0.0) {
        if (!(r->t < t_end)) { r->done = 1; return; }
        dt = jmin(dt, t_end - r->t);
    }
    // an infinite signal speed (overflowed state) gives dt = 0: time cannot
    // advance, stop and report instead of stepping in place
    if (!(dt > 0.0)) { r->done = 2; return; }
    r->dt = dt;
    r->smax = 0ull;
    r->nanflag = 0u;
}

__global__ void advance_kernel(Dev* r) {
    if (r->done) return;
    r->t += r->dt;
    r->steps += 1;
}

struct State {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
    // key of the captured graph
    double* U = nullptr;
    int nx = 0, ny = 0, nz = 0, bc = 0, prec = 0, variant = -1;
    double dx = 0, dy = 0, dz = 0, gamma = 0, cfl = 0, rho_floor = 0, P_floor = 0, t_end = 0;
    double *A = nullptr, *B = nullptr;
    Dev* r = nullptr;
    cudaStream_t cap = nullptr;   // private stream used only to capture (the caller's may be the legacy stream)
    cudaEvent_t flag_ev[2] = {nullptr, nullptr};   // done-flag readbacks of the replay chunks
};

State* state(bsn_ctx* ctx) {
    if (!ctx->run_state) ctx->run_state = new State();
    return (State*)ctx->run_state;
}

void release(State* S) {
    if (S->exec) cudaGraphExecDestroy(S->exec);
    if (S->graph) cudaGraphDestroy(S->graph);
    S->exec = nullptr;
    S->graph = nullptr;
}

}  // namespace run

void run_state_free(bsn_ctx* ctx) {
    if (!ctx->run_state) return;
    run::State* S = (run::State*)ctx->run_state;
    run::release(S);
    if (S->cap) cudaStreamDestroy(S->cap);
    for (cudaEvent_t e : S->flag_ev)
        if (e) cudaEventDestroy(e);
    delete S;
    ctx->run_state = nullptr;
}

// One RK3 step with the stencil precision `prec` (FP64 state throughout).
bsn_status rk3_prec(bsn_ctx* ctx, f64::StageArgs base, double* U, double dt, int prec) {
    Geom G(base.nx, base.ny, base.nz);
    size_t bytes = sizeof(double) * (size_t)G.nelem();
    bsn_status st;
    double* A = (double*)slot(ctx, SLOT_A, bytes, &st); BSN_TRY(st);
    double* B = (double*)slot(ctx, SLOT_B, bytes, &st); BSN_TRY(st);
    double* in[3] = {U, A, B};
    double* out[3] = {A, B, U};
    for (int s = 0; s < 3; ++s) {
        f64::StageArgs a = base;
        a.Uin = in[s]; a.Un = U; a.Uout = out[s]; a.mode = 0;
        set_stage(a, s + 1, dt);
        BSN_TRY(stage_launch(ctx, prec, a));
    }
    return f64_ghost_combine(ctx, U, B, nullptr, base.nx, base.ny, base.nz, base.bc, dt);
}

bsn_status graph_replay(bsn_ctx* ctx, cudaGraphExec_t exec, int kernels, int n_steps, bool until_done,
                        const int* done_dev, cudaEvent_t ev[2], volatile int* hflag) {
    if (!until_done) {
        for (int i = 0; i < n_steps; ++i) {
            BSN_CUDA(ctx, cudaGraphLaunch(exec, ctx->stream));
            ctx->launches += kernels;
        }
        return BSN_OK;
    }
    const int CHUNK = 16;
    for (int b = 0; b < 2; ++b)
        if (!ev[b]) BSN_CUDA(ctx, cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
    int launched = 0;
    for (int chunk = 0; launched < n_steps; ++chunk) {
        int c = std::min(CHUNK, n_steps - launched);
        for (int i = 0; i < c; ++i) {
            BSN_CUDA(ctx, cudaGraphLaunch(exec, ctx->stream));
            ctx->launches += kernels;
        }
        launched += c;
        BSN_CUDA(ctx, cudaMemcpyAsync((void*)(hflag + (chunk & 1)), done_dev, sizeof(int), cudaMemcpyDeviceToHost,
                                      ctx->stream));
        BSN_CUDA(ctx, cudaEventRecord(ev[chunk & 1], ctx->stream));
        if (chunk > 0) {
            BSN_CUDA(ctx, cudaEventSynchronize(ev[(chunk - 1) & 1]));
            if (hflag[(chunk - 1) & 1]) break;
        }
    }
    return BSN_OK;
}

}  // namespace bsn

using namespace bsn;
using namespace bsn::run;

static bsn_status check_step_args(bsn_ctx* ctx, double* U, int nx, int ny, int nz, int bc, int prec) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U) return set_err(ctx, BSN_ERR_ARG, "U is null");
    if (bc != BSN_BC_OUTFLOW && bc != BSN_BC_PERIODIC) return set_err(ctx, BSN_ERR_ARG, "bad bc %d", bc);
    if (bc == BSN_BC_PERIODIC && (nx < BSN_NG || ny < BSN_NG || nz < BSN_NG))
        return set_err(ctx, BSN_ERR_ARG, "periodic boundaries need n >= 3 per axis");
    if (prec != PREC_F64 && prec != PREC_F32 && prec != PREC_LEARNED)
        return set_err(ctx, BSN_ERR_ARG, "bad precision %d", prec);
    return BSN_OK;
}

extern "C" bsn_status bsn_euler3d_rhs_f32(bsn_ctx* ctx, double* dU, double* Fx, double* Fy, double* Fz, double* U,
                                          int nx, int ny, int nz, double dx, double dy, double dz, double gamma,
                                          int bc, double rho_floor, double P_floor, int fill_ghosts) {
    BSN_TRY(check_step_args(ctx, U, nx, ny, nz, bc, PREC_F32));
    if (!dU) return set_err(ctx, BSN_ERR_ARG, "dU is null");
    Geom G(nx, ny, nz);
    if (fill_ghosts) BSN_TRY(f64_fill_ghosts(ctx, U, nx, ny, nz, bc));
    long long X = nx + 6, Y = ny + 6, Z = nz + 6;
    if (Fx) BSN_CUDA(ctx, cudaMemsetAsync(Fx, 0, sizeof(double) * 5 * (X + 1) * Y * Z, ctx->stream));
    if (Fy) BSN_CUDA(ctx, cudaMemsetAsync(Fy, 0, sizeof(double) * 5 * X * (Y + 1) * Z, ctx->stream));
    if (Fz) BSN_CUDA(ctx, cudaMemsetAsync(Fz, 0, sizeof(double) * 5 * X * Y * (Z + 1), ctx->stream));
    BSN_CUDA(ctx, cudaMemsetAsync(dU, 0, sizeof(double) * G.nelem(), ctx->stream));
    f64::StageArgs A;
    stage_args_init(A, nx, ny, nz, dx, dy, dz, gamma, bc, rho_floor, P_floor);
    A.Uin = U;
    A.Gh = U;   // ghosts are whatever U holds (filled above or by the caller)
    A.dU = dU;
    A.F[0] = Fx; A.F[1] = Fy; A.F[2] = Fz;
    A.mode = 1;
    A.stiff_guard = ctx->stiff_guard;
    BSN_TRY(stage_launch(ctx, PREC_F32, A));
    // euler3d_rhs! floors U in place; the stage kernel floored its staged copies
    return f64_floors(ctx, U, nx, ny, nz, rho_floor, P_floor, gamma);
}

extern "C" bsn_status bsn_euler3d_step_f32(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double dx, double dy,
                                           double dz, double dt, double gamma, int bc, double rho_floor,
                                           double P_floor) {
    BSN_TRY(check_step_args(ctx, U, nx, ny, nz, bc, PREC_F32));
    f64::StageArgs A;
    stage_args_init(A, nx, ny, nz, dx, dy, dz, gamma, bc, rho_floor, P_floor);
    A.stiff_guard = ctx->stiff_guard;
    return rk3_prec(ctx, A, U, dt, PREC_F32);
}

extern "C" bsn_status bsn_euler3d_step_learned(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double dx,
                                               double dy, double dz, double dt, double gamma, int bc,
                                               double rho_floor, double P_floor) {
    BSN_TRY(check_step_args(ctx, U, nx, ny, nz, bc, PREC_LEARNED));
    f64::StageArgs A;
    stage_args_init(A, nx, ny, nz, dx, dy, dz, gamma, bc, rho_floor, P_floor);
    A.learned_split = 1;
    return rk3_prec(ctx, A, U, dt, PREC_LEARNED);
}

extern "C" bsn_status bsn_run_steps(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                                    double gamma, double cfl, int bc, double rho_floor, double P_floor, int precision,
                                    int n_steps, double t_end, double* t_inout, int* steps_done) {
    BSN_TRY(check_step_args(ctx, U, nx, ny, nz, bc, precision));
    if (!t_inout) return set_err(ctx, BSN_ERR_ARG, "t_inout is null");
    if (n_steps < 0) return set_err(ctx, BSN_ERR_ARG, "n_steps < 0");
    Geom G(nx, ny, nz);
    size_t bytes = sizeof(double) * (size_t)G.nelem();
    bsn_status st;
    double* A = (double*)slot(ctx, SLOT_A, bytes, &st); BSN_TRY(st);
    double* B = (double*)slot(ctx, SLOT_B, bytes, &st); BSN_TRY(st);
    Dev* r = (Dev*)slot(ctx, SLOT_RUN, sizeof(Dev), &st); BSN_TRY(st);
    State* S = state(ctx);

    f64::StageArgs base;
    stage_args_init(base, nx, ny, nz, dx, dy, dz, gamma, bc, rho_floor, P_floor);
    base.Uin = U; base.Un = U;
    base.learned_split = 1;   // a uniform grid: mostly uniform blocks away from the flow's features
    base.stiff_guard = ctx->stiff_guard;
    base.tune_class = TUNE_RUN;
    // autotune before any capture (it launches and times kernels)
    auto tune = [&]() -> bsn_status {
        bsn_status ts;
        double* scratch = (double*)slot(ctx, SLOT_UN, bytes, &ts); BSN_TRY(ts);
        return stage_autotune(ctx, precision, base, scratch);
    };
    BSN_TRY(tune());
    int variant = tile_code(ctx, precision, base);

    init_kernel<<<1, 1, 0, ctx->stream>>>(r, *t_inout);
    BSN_TRY(launch_check(ctx, "run_init_kernel"));
    BSN_TRY(f64_cfl_fold(ctx, U, nx, ny, nz, dx, dy, dz, gamma, &r->smax, &r->nanflag));

    bool same = S->exec && S->U == U && S->nx == nx && S->ny == ny && S->nz == nz && S->dx == dx && S->dy == dy &&
                S->dz == dz && S->gamma == gamma && S->cfl == cfl && S->bc == bc && S->rho_floor == rho_floor &&
                S->P_floor == P_floor && S->prec == precision && S->t_end == t_end && S->variant == variant &&
                S->A == A && S->B == B && S->r == r;
    auto capture = [&]() -> bsn_status {
        release(S);
        if (!S->cap) BSN_CUDA(ctx, cudaStreamCreateWithFlags(&S->cap, cudaStreamNonBlocking));
        // everything enqueued so far (init, CFL fold) happens before the first replay on ctx->stream
        bool prof = ctx->profiling;
        ctx->profiling = false;
        long long l0 = ctx->launches;
        cudaStream_t user = ctx->stream;
        ctx->stream = S->cap;
        {
            cudaError_t be = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
            if (be != cudaSuccess) { ctx->stream = user; ctx->profiling = prof; return cuda_check(ctx, be, "cudaStreamBeginCapture"); }
        }
        bsn_status cst = BSN_OK;
        dt_kernel<<<1, 1, 0, ctx->stream>>>(r, cfl, t_end);
        cst = launch_check(ctx, "run_dt_kernel");
        double* in[3] = {U, A, B};
        double* out[3] = {A, B, U};
        for (int s = 0; s < 3 && cst == BSN_OK; ++s) {
            f64::StageArgs a = base;
            a.Uin = in[s]; a.Un = U; a.Uout = out[s]; a.mode = 0;
            set_stage(a, s + 1, 0.0);
            a.dt_dev = &r->dt;
            a.done_dev = &r->done;
            if (s == 2) { a.cfl_max = &r->smax; a.cfl_nan = &r->nanflag; }
            cst = stage_launch(ctx, precision, a);
        }
        if (cst == BSN_OK) cst = f64_ghost_combine(ctx, U, B, nullptr, nx, ny, nz, bc, 0.0, &r->dt, &r->done);
        if (cst == BSN_OK) {
            advance_kernel<<<1, 1, 0, ctx->stream>>>(r);
            cst = launch_check(ctx, "run_advance_kernel");
        }
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        ctx->stream = user;
        ctx->profiling = prof;
        S->kernels = (int)(ctx->launches - l0);
        ctx->launches = l0;
        if (cst != BSN_OK) { if (g) cudaGraphDestroy(g); return cst; }
        BSN_CUDA(ctx, e);
        S->graph = g;
        BSN_CUDA(ctx, cudaGraphInstantiate(&S->exec, g, 0));
        S->U = U; S->nx = nx; S->ny = ny; S->nz = nz; S->dx = dx; S->dy = dy; S->dz = dz; S->gamma = gamma;
        S->cfl = cfl; S->bc = bc; S->rho_floor = rho_floor; S->P_floor = P_floor; S->prec = precision;
        S->t_end = t_end; S->variant = variant; S->A = A; S->B = B; S->r = r;
        return BSN_OK;
    };
    if (!same) BSN_TRY(capture());
    double* h = (double*)pinned(ctx, 128, &st); BSN_TRY(st);
    // replays after t_end are no-ops: with t_end, stop once the device says done
    const bool settle = n_steps >= 2 && !tile_settled(ctx, TUNE_RUN, precision);
    BSN_TRY(graph_replay(ctx, S->exec, S->kernels, settle ? 1 : n_steps, t_end > 0.0, &r->done, S->flag_ev,
                         (volatile int*)(h + 8)));
    if (settle) {   // the tile re-timed on the state after the first step
        BSN_TRY(tile_retime(ctx, TUNE_RUN, precision, tune));
        if (tile_code(ctx, precision, base) != variant) {
            variant = tile_code(ctx, precision, base);
            BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            BSN_TRY(capture());
        }
        BSN_TRY(graph_replay(ctx, S->exec, S->kernels, n_steps - 1, t_end > 0.0, &r->done, S->flag_ev,
                             (volatile int*)(h + 8)));
    }
    BSN_CUDA(ctx, cudaMemcpyAsync(h, r, sizeof(Dev), cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    Dev d;
    memcpy(&d, h, sizeof(Dev));
    *t_inout = d.t;
    if (steps_done) *steps_done = d.steps;
    if (d.done == 2) return set_err(ctx, BSN_ERR_NONFINITE, "time step collapsed to 0 at t = %.17g (infinite signal speed)", d.t);
    return BSN_OK;
}
