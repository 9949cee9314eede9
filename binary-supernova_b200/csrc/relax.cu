// relax.cu -- relax_ic! (src/relax_ic.jl:200-330) on the device: SSP-RK3
// steps whose stages carry the hydro RHS, BH gravity (BHs held fixed),
// optional self-gravity (a Poisson solve per stage, as add_self_gravity_source!),
// the rotating-frame forces (Omega != 0) and velocity damping toward rest,
// until t_max, KE/E_thermal < KE_tol, or the kinetic-energy ratio turns back
// up past its post-peak minimum.  dt, t, the ratio and its running peak and
// minimum stay in device memory; each step is one CUDA graph and the stop
// rule is evaluated by a one-thread kernel, so the host does not read the
// state between steps.  Built with -fmad=false (the FP64 stencils and
// sources are the reference's operations in its order).
#include <cmath>
#include <cstring>

#include "diagnostics.cuh"
#include "poisson.cuh"
#include "stage_launch.cuh"

namespace bsn {
namespace relax {

struct Dev {
    double dt, t;
    unsigned long long smax;   // CFL maximum of the step's result (double bits)
    unsigned int nanflag;
    int done, steps, descended, pad;
    double ke_ratio, ke_peak, ke_valley;
    double tot[diag::NDIAG];   // diagnostics of the end-of-step state
};

__global__ void init_kernel(Dev* r) {
    r->dt = 0.0; r->t = 0.0; r->smax = 0ull; r->nanflag = 0u; r->done = 0; r->steps = 0; r->descended = 0;
    r->ke_ratio = INFINITY; r->ke_peak = 0.0; r->ke_valley = INFINITY;
}

// loop head `while t < t_max && KE_ratio > KE_tol`, then
// dt = min(cfl_dt_3d(U, ...), t_max - t)
__global__ void dt_kernel(Dev* r, double cfl, double t_max, double ke_tol) {
    if (r->done) return;
    if (!(r->t < t_max && r->ke_ratio > ke_tol)) { r->done = 1; return; }
    double smax = __longlong_as_double((long long)r->smax);
    double dt = r->nanflag ? INFINITY : (smax > 0.0 ? cfl / smax : INFINITY);
    dt = jmin(dt, t_max - r->t);
    if (!(dt > 0.0)) { r->done = 2; return; }
    r->dt = dt;
    r->smax = 0ull;
    r->nanflag = 0u;
}

// after the step: t += dt, n_steps += 1, KE_ratio = KE / max(E - KE, 0) and
// the peak / post-peak-minimum stop (src/relax_ic.jl:300-318)
__global__ void check_kernel(Dev* r) {
    if (r->done) return;
    r->t += r->dt;
    r->steps += 1;
    const double E = r->tot[0], KE = r->tot[1];
    const double Eth = jmax(E - KE, 0.0);
    const double kr = Eth > 0.0 ? KE / Eth : 0.0;
    r->ke_ratio = kr;
    r->ke_peak = jmax(r->ke_peak, kr);
    if (!r->descended) r->descended = kr < 0.9 * r->ke_peak;
    if (r->descended) {
        r->ke_valley = jmin(r->ke_valley, kr);
        if (kr > 1.1 * r->ke_valley) r->done = 1;
    }
}

struct State {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
    std::vector<double> key;
    cudaStream_t cap = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
};

}  // namespace relax

void relax_state_free(bsn_ctx* ctx) {
    if (!ctx->relax_state) return;
    relax::State* S = (relax::State*)ctx->relax_state;
    S->release();
    if (S->cap) cudaStreamDestroy(S->cap);
    for (cudaEvent_t e : S->ev)
        if (e) cudaEventDestroy(e);
    delete S;
    ctx->relax_state = nullptr;
}

}  // namespace bsn

using namespace bsn;
using namespace bsn::relax;

extern "C" bsn_status bsn_relax_ic(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                                   double gamma, const bsn_bh* bhs, int nbh, double x0, double y0, double z0,
                                   double t_damp, double t_max, double cfl, double rho_floor, double P_floor,
                                   double KE_tol, double Omega, int self_gravity, int precision, int max_steps,
                                   double* t_out, int* n_steps_out, double* ke_ratio_out) {
    if (!ctx) return BSN_ERR_ARG;
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || (nbh > 0 && !bhs)) return set_err(ctx, BSN_ERR_ARG, "null argument");
    if (nbh < 0 || nbh > f64::MAXBH) return set_err(ctx, BSN_ERR_UNSUPPORTED, "at most %d black holes", f64::MAXBH);
    if (!(t_damp > 0.0)) return set_err(ctx, BSN_ERR_ARG, "t_damp must be positive");
    if (max_steps < 0) return set_err(ctx, BSN_ERR_ARG, "max_steps < 0");
    if (precision != PREC_F64 && precision != PREC_F32 && precision != PREC_LEARNED)
        return set_err(ctx, BSN_ERR_ARG, "bad precision %d", precision);
    Geom G(nx, ny, nz);
    size_t bytes = sizeof(double) * (size_t)G.nelem();
    bsn_status st;
    double* A = (double*)slot(ctx, SLOT_A, bytes, &st); BSN_TRY(st);
    double* B = (double*)slot(ctx, SLOT_B, bytes, &st); BSN_TRY(st);
    Dev* r = (Dev*)slot(ctx, SLOT_RELAX, sizeof(Dev), &st); BSN_TRY(st);
    double* part = (double*)slot(ctx, SLOT_DIAGREC, sizeof(double) * 2 * diag::NDIAG * diag::BLOCKS, &st);
    BSN_TRY(st);
    double* phi = nullptr;
    if (self_gravity) {
        phi = (double*)slot(ctx, SLOT_PHI, sizeof(double) * (size_t)nx * ny * nz, &st); BSN_TRY(st);
        if (precision == PREC_F64) BSN_TRY(poisson_prepare(ctx, nx, ny, nz, dx, dy, dz));
        else BSN_TRY(poisson_prepare_f32(ctx, nx, ny, nz, dx, dy, dz));
    }
    // the stage arguments: outflow hydro, BH gravity of the fixed BHs, the
    // rotating frame when Omega != 0, damping toward rest (the driver passes
    // Omega = 0 to relax_damping_source!)
    f64::StageArgs base;
    stage_args_init(base, nx, ny, nz, dx, dy, dz, gamma, BSN_BC_OUTFLOW, rho_floor, P_floor);
    base.stiff_guard = ctx->stiff_guard;
    base.x0 = x0; base.y0 = y0; base.z0 = z0;
    if (nbh > 0) {
        base.use_bh = 1;
        base.bh.n = nbh;
        for (int i = 0; i < nbh; ++i) {
            base.bh.px[i] = bhs[i].pos[0]; base.bh.py[i] = bhs[i].pos[1]; base.bh.pz[i] = bhs[i].pos[2];
            base.bh.mass[i] = bhs[i].mass; base.bh.eps[i] = bhs[i].eps;
        }
    }
    if (Omega != 0.0) { base.use_rot = 1; base.rot_omega = Omega; }
    base.use_damp = 1;
    base.damp_t = t_damp;
    base.damp_inv_td = 1.0 / t_damp;
    base.damp_omega = 0.0;
    base.tune_class = TUNE_RELAX;
    {
        f64::StageArgs p = base;
        p.Uin = U;
        double* scratch = (double*)slot(ctx, SLOT_UN, bytes, &st); BSN_TRY(st);
        BSN_TRY(stage_autotune(ctx, precision, p, scratch));
    }
    const int variant = tile_code(ctx, precision, base);

    init_kernel<<<1, 1, 0, ctx->stream>>>(r);
    BSN_TRY(launch_check(ctx, "relax_init_kernel"));
    BSN_TRY(f64_cfl_fold(ctx, U, nx, ny, nz, dx, dy, dz, gamma, &r->smax, &r->nanflag));

    if (!ctx->relax_state) ctx->relax_state = new State();
    State* S = (State*)ctx->relax_state;
    std::vector<double> key = {(double)(uintptr_t)U, (double)nx, (double)ny, (double)nz, dx, dy, dz, gamma,
                               (double)nbh, x0, y0, z0, t_damp, t_max, cfl, rho_floor, P_floor, KE_tol, Omega,
                               (double)self_gravity, (double)precision, (double)variant, (double)(uintptr_t)A,
                               (double)(uintptr_t)B, (double)(uintptr_t)r, (double)(uintptr_t)part,
                               (double)(uintptr_t)phi};
    for (int i = 0; i < nbh; ++i)
        key.insert(key.end(), {bhs[i].pos[0], bhs[i].pos[1], bhs[i].pos[2], bhs[i].mass, bhs[i].eps});
    if (!(S->exec && S->key == key)) {
        S->release();
        if (!S->cap) BSN_CUDA(ctx, cudaStreamCreateWithFlags(&S->cap, cudaStreamNonBlocking));
        bool prof = ctx->profiling;
        ctx->profiling = false;
        long long l0 = ctx->launches;
        cudaStream_t user = ctx->stream;
        ctx->stream = S->cap;
        cudaError_t be = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        if (be != cudaSuccess) { ctx->stream = user; ctx->profiling = prof; return cuda_check(ctx, be, "cudaStreamBeginCapture"); }
        auto body = [&]() -> bsn_status {
            dt_kernel<<<1, 1, 0, ctx->stream>>>(r, cfl, t_max, KE_tol);
            BSN_TRY(launch_check(ctx, "relax_dt_kernel"));
            double* in[3] = {U, A, B};
            double* out[3] = {A, B, U};
            for (int s = 0; s < 3; ++s) {
                f64::StageArgs a = base;
                a.Uin = in[s]; a.Un = U; a.Uout = out[s]; a.mode = 0;
                set_stage(a, s + 1, 0.0);
                a.dt_dev = &r->dt;
                a.done_dev = &r->done;
                if (self_gravity) {
                    if (precision == PREC_F64)
                        BSN_TRY(poisson_from_state(ctx, in[s], nx, ny, nz, dx, dy, dz, rho_floor, phi));
                    else
                        BSN_TRY(poisson_from_state_f32(ctx, in[s], nx, ny, nz, dx, dy, dz, rho_floor, phi));
                    a.phi = phi; a.use_sg = 1;
                }
                if (s == 2) { a.cfl_max = &r->smax; a.cfl_nan = &r->nanflag; }
                BSN_TRY(stage_launch(ctx, precision, a));
            }
            BSN_TRY(f64_ghost_combine(ctx, U, B, nullptr, nx, ny, nz, BSN_BC_OUTFLOW, 0.0, &r->dt, &r->done));
            // gas_energy_total and gas_kinetic_total of the new state (one reduction)
            BSN_TRY(diag::launch(ctx, U, nx, ny, nz, dx, dy, dz, x0, y0, z0, nullptr, nullptr, 0, gamma, part,
                                 r->tot, nullptr, nullptr, nullptr, &r->done, 0));
            check_kernel<<<1, 1, 0, ctx->stream>>>(r);
            return launch_check(ctx, "relax_check_kernel");
        };
        bsn_status cst = body();
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        ctx->stream = user;
        ctx->profiling = prof;
        S->kernels = (int)(ctx->launches - l0);
        ctx->launches = l0;
        if (cst != BSN_OK) { if (graph) cudaGraphDestroy(graph); return cst; }
        BSN_CUDA(ctx, e);
        S->graph = graph;
        BSN_CUDA(ctx, cudaGraphInstantiate(&S->exec, graph, 0));
        S->key = key;
    }
    double* h = (double*)pinned(ctx, sizeof(Dev) + 128, &st); BSN_TRY(st);
    BSN_TRY(graph_replay(ctx, S->exec, S->kernels, max_steps, true, &r->done, S->ev,
                         (volatile int*)((char*)h + sizeof(Dev))));
    BSN_CUDA(ctx, cudaMemcpyAsync(h, r, sizeof(Dev), cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    Dev d;
    memcpy(&d, h, sizeof(Dev));
    if (t_out) *t_out = d.t;
    if (n_steps_out) *n_steps_out = d.steps;
    if (ke_ratio_out) *ke_ratio_out = d.ke_ratio;
    if (d.done == 2)
        return set_err(ctx, BSN_ERR_NONFINITE, "time step collapsed to 0 at t = %.17g (infinite signal speed)", d.t);
    return BSN_OK;
}
