// coupled_run.cu -- the production driver loop on the device: dt = CFL (capped
// by dt_max, clamped to t_end), then coupled_step! (scripts/run_sn50_fiducial.jl
// :756-818) -- gas force on every BH, the BH orbit (nbody_step!, FP64), the
// SSP-RK3 stages with BH gravity, self-gravity and sinks in the driver's order,
// accrete! on every active sink -- with the BHs, t and dt kept in device
// memory and each step one CUDA graph.  Built with -fmad=false: the FP64
// orbit, accretion and source arithmetic are the same operations in the same
// order as the host versions (src/nbody.jl:24-104, src/sinks.jl:74-109).
#include <cmath>
#include <cstring>

#include "hydro_f64.cuh"
#include "diagnostics.cuh"
#include "poisson.cuh"
#include "stage_launch.cuh"
#include "fmr_nested.cuh"
#include "sums.cuh"

namespace bsn {
namespace crun {

using f64::MAXBH;

struct Dev {
    double dt, t;
    unsigned long long smax;
    unsigned int nanflag;
    int done, steps;
    int nbh, pad;
    bsn_bh bh[MAXBH];
    double Fg[3 * MAXBH];
    f64::BHSrc bsrc;
    f64::SinkSrc ssrc;
    // mass ledger: per-stage sums of the step being taken, per level (the
    // stage kernels add, f64_ledger_fold clears), and the totals since the
    // start of the call (f64::LEDT_*)
    double led[f64::MAXLEV][3][f64::LED_TERMS];
    double led_tot[f64::LEDT_COUNT];
};

__global__ void init_kernel(Dev* r, double t, const bsn_bh* bhs, int nbh) {
    r->dt = 0.0; r->t = t; r->smax = 0ull; r->nanflag = 0u; r->done = 0; r->steps = 0; r->nbh = nbh;
    for (int i = 0; i < nbh; ++i) r->bh[i] = bhs[i];
    for (int i = 0; i < 3 * MAXBH; ++i) r->Fg[i] = 0.0;
    for (int l = 0; l < f64::MAXLEV; ++l)
        for (int s = 0; s < 3; ++s)
            for (int q = 0; q < f64::LED_TERMS; ++q) r->led[l][s][q] = 0.0;
    for (int q = 0; q < f64::LEDT_COUNT; ++q) r->led_tot[q] = 0.0;
}

// dt = cfl / max speed (Inf for NaN or zero), capped by dt_max > 0, clamped to t_end > 0.
__global__ void dt_kernel(Dev* r, double cfl, double t_end, double dt_max) {
    if (r->done) return;
    double smax = __longlong_as_double((long long)r->smax);
    double dt = r->nanflag ? INFINITY : (smax > 0.0 ? cfl / smax : INFINITY);
    if (dt_max > 0.0) dt = jmin(dt, dt_max);
    if (t_end > 0.0) {
        if (!(r->t < t_end)) { r->done = 1; return; }
        dt = jmin(dt, t_end - r->t);
    }
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

// gas_force_on_bh partial sums for BH i (compensated, as f64::gas_force_kernel)
using sums::DD;
using sums::dd_add;
using sums::dd_merge;

// active cells [lo, hi] (0-based, inclusive per axis) left out of a sum: the
// region a finer level covers; lo > hi leaves nothing out
struct Box {
    int lo[3], hi[3];
};

__global__ void gas_force_kernel(const double* U, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                                 double y0, double z0, const Dev* r, int i, double* part, Box skip) {
    if (r->done) return;
    const bsn_bh bh = r->bh[i];
    Geom G(nx, ny, nz);
    double dV = dx * dy * dz;
    DD s[3] = {{0, 0}, {0, 0}, {0, 0}};
    long long n = (long long)nx * ny * nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int a = (int)(t % nx); long long rr = t / nx; int b = (int)(rr % ny); int c = (int)(rr / ny);
        if (a >= skip.lo[0] && a <= skip.hi[0] && b >= skip.lo[1] && b <= skip.hi[1] && c >= skip.lo[2] &&
            c <= skip.hi[2])
            continue;
        double xc, yc, zc;
        f64::cell_xyz(a, b, c, x0, y0, z0, dx, dy, dz, xc, yc, zc);
        double ddx = xc - bh.pos[0], ddy = yc - bh.pos[1], ddz = zc - bh.pos[2];
        double r2 = sq(ddx) + sq(ddy) + sq(ddz) + sq(bh.eps);
        double r3 = r2 * sqrt(r2);
        double fac = bh.mass / r3 * U[G.act(a, b, c)] * dV;
        dd_add(s[0], fac * ddx);
        dd_add(s[1], fac * ddy);
        dd_add(s[2], fac * ddz);
    }
    __shared__ DD red[3][32];
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o > 0; o >>= 1) {
            DD other = {__shfl_xor_sync(0xffffffffu, s[d].hi, o), __shfl_xor_sync(0xffffffffu, s[d].lo, o)};
            s[d] = dd_merge(s[d], other);
        }
        if ((threadIdx.x & 31) == 0) red[d][threadIdx.x >> 5] = s[d];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int d = 0; d < 3; ++d) {
            DD acc = red[d][0];
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) acc = dd_merge(acc, red[d][w]);
            part[6 * blockIdx.x + 2 * d] = acc.hi;
            part[6 * blockIdx.x + 2 * d + 1] = acc.lo;
        }
    }
}

// total of BH i's partials, zeroed when non-finite or above 1e3 in norm (the
// driver's guard, scripts/run_sn50_fiducial.jl:765-769)
__global__ void gas_force_finish(const double* part, int nblocks, Dev* r, int i) {
    if (r->done || blockIdx.x != 0) return;
    double F[3];
    sums::merge_partials3<256>(part, nblocks, F);
    if (threadIdx.x != 0) return;
    bool fin = isfinite(F[0]) && isfinite(F[1]) && isfinite(F[2]);
    if (!fin || sqrt(F[0] * F[0] + F[1] * F[1] + F[2] * F[2]) > 1e3) F[0] = F[1] = F[2] = 0.0;
    for (int d = 0; d < 3; ++d) r->Fg[3 * i + d] = F[d];
}

// nbody_step! (src/nbody.jl:24-104): SSP-RK3 of the BHs with frozen gas force
__device__ void nbody_rhs(double (*dp)[3], double (*dv)[3], const bsn_bh* b, int n, const double* Fg) {
    for (int i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) dp[i][d] = b[i].vel[d];
        double a[3] = {Fg[3 * i] / b[i].mass, Fg[3 * i + 1] / b[i].mass, Fg[3 * i + 2] / b[i].mass};
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            double x = b[j].pos[0] - b[i].pos[0], y = b[j].pos[1] - b[i].pos[1], z = b[j].pos[2] - b[i].pos[2];
            double r2 = x * x + y * y + z * z + b[j].eps * b[j].eps;
            double r3 = r2 * sqrt(r2);
            double fac = b[j].mass / r3;
            a[0] = a[0] + fac * x; a[1] = a[1] + fac * y; a[2] = a[2] + fac * z;
        }
        for (int d = 0; d < 3; ++d) dv[i][d] = a[d];
    }
}

__global__ void nbody_kernel(Dev* r) {
    if (r->done || threadIdx.x != 0 || blockIdx.x != 0) return;
    const int n = r->nbh;
    bsn_bh* b = r->bh;
    bool ok = n > 0;
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) ok = ok && isfinite(b[i].pos[d]) && isfinite(b[i].vel[d]);
    if (!ok) return;
    const double dt = r->dt;
    double p0[MAXBH][3], v0[MAXBH][3], p1[MAXBH][3], v1[MAXBH][3], p2[MAXBH][3], v2[MAXBH][3], DP[MAXBH][3],
        DV[MAXBH][3];
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) { p0[i][d] = b[i].pos[d]; v0[i][d] = b[i].vel[d]; }
    nbody_rhs(DP, DV, b, n, r->Fg);   // stage 1
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            p1[i][d] = p0[i][d] + dt * DP[i][d];
            v1[i][d] = v0[i][d] + dt * DV[i][d];
            b[i].pos[d] = p1[i][d]; b[i].vel[d] = v1[i][d];
        }
    nbody_rhs(DP, DV, b, n, r->Fg);   // stage 2
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            p2[i][d] = 0.75 * p0[i][d] + 0.25 * (p1[i][d] + dt * DP[i][d]);
            v2[i][d] = 0.75 * v0[i][d] + 0.25 * (v1[i][d] + dt * DV[i][d]);
        }
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) { b[i].pos[d] = p2[i][d]; b[i].vel[d] = v2[i][d]; }
    nbody_rhs(DP, DV, b, n, r->Fg);   // stage 3
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            b[i].pos[d] = (1.0 / 3.0) * p0[i][d] + (2.0 / 3.0) * (p2[i][d] + dt * DP[i][d]);
            b[i].vel[d] = (1.0 / 3.0) * v0[i][d] + (2.0 / 3.0) * (v2[i][d] + dt * DV[i][d]);
        }
}

// r_sink, t_sink (src/BinarySupernova.jl:159-171)
__device__ __forceinline__ double r_sink(const bsn_bh& b) { return jmax(6.0 * b.mass / (b.c_code * b.c_code), b.r_floor); }
__device__ __forceinline__ double t_sink(const bsn_bh& b, double f_sink) {
    double rs = r_sink(b);
    double v_ff = sqrt(2.0 * b.mass / rs);
    return f_sink * rs / v_ff;
}

// the stage sources of the step from the (updated) BHs: gravity of all,
// sinks of the first BH before t_bh2_sink_on and of all after
__global__ void fill_kernel(Dev* r, double f_sink, int torque_free, double rho_min, double t_bh2_sink_on) {
    if (r->done || threadIdx.x != 0 || blockIdx.x != 0) return;
    const int n = r->nbh;
    const int ns = (r->t < t_bh2_sink_on) ? (n < 1 ? n : 1) : n;
    f64::BHSrc& B = r->bsrc;
    f64::SinkSrc& S = r->ssrc;
    B.n = n;
    S.n = ns; S.torque_free = torque_free ? 1 : 0; S.rho_min = rho_min;
    for (int i = 0; i < MAXBH; ++i) {
        const bool on = i < n;
        B.px[i] = on ? r->bh[i].pos[0] : 0.0; B.py[i] = on ? r->bh[i].pos[1] : 0.0; B.pz[i] = on ? r->bh[i].pos[2] : 0.0;
        B.mass[i] = on ? r->bh[i].mass : 0.0; B.eps[i] = on ? r->bh[i].eps : 0.0;
        const bool sk = i < ns;
        S.px[i] = sk ? r->bh[i].pos[0] : 0.0; S.py[i] = sk ? r->bh[i].pos[1] : 0.0; S.pz[i] = sk ? r->bh[i].pos[2] : 0.0;
        S.vx[i] = sk ? r->bh[i].vel[0] : 0.0; S.vy[i] = sk ? r->bh[i].vel[1] : 0.0; S.vz[i] = sk ? r->bh[i].vel[2] : 0.0;
        S.rs[i] = sk ? r_sink(r->bh[i]) : 0.0; S.ts[i] = sk ? t_sink(r->bh[i], f_sink) : 0.0;
    }
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// accrete! (src/sinks.jl:74-109) for sink i from the end-of-step state, summed
// in the reference's (k, j, i) order over the sphere's index box, one thread
__global__ void accrete_kernel(const double* U, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                               double y0, double z0, Dev* r, int i, double f_sink, double rho_min) {
    if (r->done || blockIdx.x != 0) return;
    if (i >= r->ssrc.n) return;
    bsn_bh& bh = r->bh[i];
    const double rs = r_sink(bh), ts = t_sink(bh, f_sink);
    const double dV = dx * dy * dz;
    const double rate = dV / ts * r->dt;
    int ilo = clampi((int)floor((bh.pos[0] - rs - x0) / dx) - 2, 0, nx - 1);
    int ihi = clampi((int)ceil((bh.pos[0] + rs - x0) / dx) + 2, 0, nx - 1);
    int jlo = clampi((int)floor((bh.pos[1] - rs - y0) / dy) - 2, 0, ny - 1);
    int jhi = clampi((int)ceil((bh.pos[1] + rs - y0) / dy) + 2, 0, ny - 1);
    int klo = clampi((int)floor((bh.pos[2] - rs - z0) / dz) - 2, 0, nz - 1);
    int khi = clampi((int)ceil((bh.pos[2] + rs - z0) / dz) + 2, 0, nz - 1);
    if (!isfinite(rs) || !isfinite(bh.pos[0]) || !isfinite(bh.pos[1]) || !isfinite(bh.pos[2])) {
        ilo = 0; ihi = nx - 1; jlo = 0; jhi = ny - 1; klo = 0; khi = nz - 1;
    }
    double v[4];
    sums::sink_sums<256>(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, bh.pos[0], bh.pos[1], bh.pos[2], rs, rate, rho_min,
                         ilo, ihi, jlo, jhi, klo, khi, v);
    if (threadIdx.x != 0) return;
    const double dm = v[0];
    if (dm > 0.0) {
        r->led_tot[f64::LEDT_ACCRETED] += dm;
        double M_new = bh.mass + dm;
        bh.vel[0] = (bh.mass * bh.vel[0] + v[1]) / M_new;
        bh.vel[1] = (bh.mass * bh.vel[1] + v[2]) / M_new;
        bh.vel[2] = (bh.mass * bh.vel[2] + v[3]) / M_new;
        bh.mass = M_new;
    }
}

struct State {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
    // key of the captured graph
    double* U = nullptr;
    int nx = 0, ny = 0, nz = 0, nbh = -1, prec = -1, variant = -1, sg = 0, torque_free = 0, evolve = 0;
    double dx = 0, x0 = 0, y0 = 0, z0 = 0, gamma = 0, cfl = 0, dt_max = 0, f_sink = 0, rho_floor = 0, P_floor = 0,
           t_on = 0, rho_min = 0, t_end = 0;
    const void* ptrs[7] = {};
    int diag_cap = 0;
    cudaStream_t cap = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
};

}  // namespace crun

void coupled_run_state_free(bsn_ctx* ctx) {
    if (!ctx->coupled_run_state) return;
    crun::State* S = (crun::State*)ctx->coupled_run_state;
    S->release();
    if (S->cap) cudaStreamDestroy(S->cap);
    for (cudaEvent_t e : S->ev)
        if (e) cudaEventDestroy(e);
    delete S;
    ctx->coupled_run_state = nullptr;
}

}  // namespace bsn

using namespace bsn;
using namespace bsn::crun;

extern "C" bsn_status bsn_coupled_run_steps(bsn_ctx* ctx, double* U, bsn_bh* bhs, int nbh, int nx, int ny, int nz,
                                            double dx, double x0, double y0, double z0, double gamma, double cfl,
                                            double dt_max, double f_sink, double rho_floor, double P_floor,
                                            int torque_free, int self_gravity, double t_bh2_sink_on,
                                            double rho_sink_min, int evolve_orbit, int precision, int n_steps,
                                            double t_end, double* t_inout, int* steps_done, double* diag_out,
                                            int diag_cap) {
    if (!ctx) return BSN_ERR_ARG;
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || !t_inout || (nbh > 0 && !bhs)) return set_err(ctx, BSN_ERR_ARG, "null argument");
    if (nbh < 0 || nbh > MAXBH) return set_err(ctx, BSN_ERR_UNSUPPORTED, "at most %d black holes", MAXBH);
    if (n_steps < 0) return set_err(ctx, BSN_ERR_ARG, "n_steps < 0");
    if (diag_out && diag_cap < 0) return set_err(ctx, BSN_ERR_ARG, "diag_cap < 0");
    if (!diag_out) diag_cap = 0;
    if (precision != PREC_F64 && precision != PREC_F32 && precision != PREC_LEARNED)
        return set_err(ctx, BSN_ERR_ARG, "bad precision %d", precision);
    Geom G(nx, ny, nz);
    size_t bytes = sizeof(double) * (size_t)G.nelem();
    bsn_status st;
    double* A = (double*)slot(ctx, SLOT_A, bytes, &st); BSN_TRY(st);
    double* B = (double*)slot(ctx, SLOT_B, bytes, &st); BSN_TRY(st);
    Dev* r = (Dev*)slot(ctx, SLOT_CRUN, sizeof(Dev), &st); BSN_TRY(st);
    const int blocks = 148 * 4;
    double* part = (double*)slot(ctx, SLOT_CRED, sizeof(double) * 6 * blocks, &st); BSN_TRY(st);
    double* dpart = nullptr;
    if (diag_out) {
        dpart = (double*)slot(ctx, SLOT_DIAGREC, sizeof(double) * 2 * diag::NDIAG * diag::BLOCKS, &st); BSN_TRY(st);
    }
    double* phi = nullptr;
    if (self_gravity) {
        phi = (double*)slot(ctx, SLOT_PHI, sizeof(double) * (size_t)nx * ny * nz, &st); BSN_TRY(st);
        if (precision == PREC_F64) BSN_TRY(poisson_prepare(ctx, nx, ny, nz, dx, dx, dx));
        else BSN_TRY(poisson_prepare_f32(ctx, nx, ny, nz, dx, dx, dx));
    }

    f64::StageArgs base;
    stage_args_init(base, nx, ny, nz, dx, dx, dx, gamma, BSN_BC_OUTFLOW, rho_floor, P_floor);
    base.x0 = x0; base.y0 = y0; base.z0 = z0;
    base.Uin = U; base.Un = U;
    base.stiff_guard = 1;   // near-vacuum cells beside the sinks: stiff FP32 faces in FP64
    base.tune_class = TUNE_COUPLED;

    // BHs to the device (through the context's pinned buffer, sized once for the
    // whole call: BH staging now, the step counters and flags later), initial CFL fold
    double* h = (double*)pinned(ctx, sizeof(Dev) + 128, &st); BSN_TRY(st);
    bsn_bh* hb = (bsn_bh*)h;
    for (int i = 0; i < nbh; ++i) hb[i] = bhs[i];
    bsn_bh* db = (bsn_bh*)part;   // staging for the initial BHs (overwritten by the step's reductions)
    BSN_CUDA(ctx, cudaMemcpyAsync(db, hb, sizeof(bsn_bh) * (nbh > 0 ? nbh : 1), cudaMemcpyHostToDevice, ctx->stream));
    init_kernel<<<1, 1, 0, ctx->stream>>>(r, *t_inout, db, nbh);
    BSN_TRY(launch_check(ctx, "coupled_init_kernel"));
    BSN_TRY(f64_cfl_fold(ctx, U, nx, ny, nz, dx, dx, dx, gamma, &r->smax, &r->nanflag));

    // tile choice before any capture, timed on stage-1 work with this loop's
    // sources (the step graph fills them again; Phi is recomputed every stage)
    auto tune = [&]() -> bsn_status {
        f64::StageArgs p = base;
        if (nbh > 0) {
            fill_kernel<<<1, 32, 0, ctx->stream>>>(r, f_sink, torque_free, rho_sink_min, t_bh2_sink_on);
            BSN_TRY(launch_check(ctx, "coupled_fill_kernel"));
            p.use_bh = 1; p.bh_dev = &r->bsrc; p.use_sink = 1; p.sk_dev = &r->ssrc;
        }
        if (self_gravity) {
            if (precision == PREC_F64) BSN_TRY(poisson_from_state(ctx, U, nx, ny, nz, dx, dx, dx, rho_floor, phi));
            else BSN_TRY(poisson_from_state_f32(ctx, U, nx, ny, nz, dx, dx, dx, rho_floor, phi));
            p.phi = phi; p.use_sg = 1;
        }
        bsn_status ts;
        double* scratch = (double*)slot(ctx, SLOT_UN, bytes, &ts); BSN_TRY(ts);
        return stage_autotune(ctx, precision, p, scratch);
    };
    BSN_TRY(tune());
    int variant = tile_code(ctx, precision, base);

    if (!ctx->coupled_run_state) ctx->coupled_run_state = new State();
    State* S = (State*)ctx->coupled_run_state;
    const void* ptrs[7] = {A, B, r, part, phi, diag_out, dpart};
    bool same = S->exec && S->U == U && S->nx == nx && S->ny == ny && S->nz == nz && S->nbh == nbh &&
                S->prec == precision && S->variant == variant && S->sg == self_gravity &&
                S->torque_free == torque_free && S->evolve == evolve_orbit && S->dx == dx && S->x0 == x0 &&
                S->y0 == y0 && S->z0 == z0 && S->gamma == gamma && S->cfl == cfl && S->dt_max == dt_max &&
                S->f_sink == f_sink && S->rho_floor == rho_floor && S->P_floor == P_floor &&
                S->t_on == t_bh2_sink_on && S->rho_min == rho_sink_min && S->t_end == t_end &&
                S->diag_cap == diag_cap && memcmp(S->ptrs, ptrs, sizeof(ptrs)) == 0;
    auto capture = [&]() -> bsn_status {
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
            dt_kernel<<<1, 1, 0, ctx->stream>>>(r, cfl, t_end, dt_max);
            BSN_TRY(launch_check(ctx, "coupled_dt_kernel"));
            // gas force on every BH from the start-of-step state, then the orbit
            for (int i = 0; i < nbh; ++i) {
                gas_force_kernel<<<blocks, 256, 0, ctx->stream>>>(U, nx, ny, nz, dx, dx, dx, x0, y0, z0, r, i, part,
                                                                  Box{{1, 1, 1}, {0, 0, 0}});
                BSN_TRY(launch_check(ctx, "coupled_gas_force_kernel"));
                gas_force_finish<<<1, 256, 0, ctx->stream>>>(part, blocks, r, i);
                BSN_TRY(launch_check(ctx, "coupled_gas_force_finish"));
            }
            if (evolve_orbit && nbh > 0) {
                nbody_kernel<<<1, 32, 0, ctx->stream>>>(r);
                BSN_TRY(launch_check(ctx, "coupled_nbody_kernel"));
            }
            fill_kernel<<<1, 32, 0, ctx->stream>>>(r, f_sink, torque_free, rho_sink_min, t_bh2_sink_on);
            BSN_TRY(launch_check(ctx, "coupled_fill_kernel"));
            // SSP-RK3 with the sources in the driver's order (stage epilogue)
            double* in[3] = {U, A, B};
            double* out[3] = {A, B, U};
            for (int s = 0; s < 3; ++s) {
                f64::StageArgs a = base;
                a.Uin = in[s]; a.Un = U; a.Uout = out[s]; a.mode = 0;
                set_stage(a, s + 1, 0.0);
                a.dt_dev = &r->dt;
                a.done_dev = &r->done;
                if (nbh > 0) { a.use_bh = 1; a.bh_dev = &r->bsrc; a.use_sink = 1; a.sk_dev = &r->ssrc; }
                if (self_gravity) {
                    if (precision == PREC_F64) BSN_TRY(poisson_from_state(ctx, in[s], nx, ny, nz, dx, dx, dx, rho_floor, phi));
                    else BSN_TRY(poisson_from_state_f32(ctx, in[s], nx, ny, nz, dx, dx, dx, rho_floor, phi));
                    a.phi = phi; a.use_sg = 1;
                }
                if (s == 2) { a.cfl_max = &r->smax; a.cfl_nan = &r->nanflag; }
                a.ledger = &r->led[0][s][0];
                a.led_bnd = 1;
                BSN_TRY(stage_launch(ctx, precision, a));
            }
            BSN_TRY(f64_ledger_fold(ctx, &r->led[0][0][0], r->led_tot, &r->dt, &r->done));
            BSN_TRY(f64_ghost_combine(ctx, U, B, nullptr, nx, ny, nz, BSN_BC_OUTFLOW, 0.0, &r->dt, &r->done));
            for (int i = 0; i < nbh; ++i) {
                accrete_kernel<<<1, 256, 0, ctx->stream>>>(U, nx, ny, nz, dx, dx, dx, x0, y0, z0, r, i, f_sink,
                                                          rho_sink_min);
                BSN_TRY(launch_check(ctx, "coupled_accrete_kernel"));
            }
            advance_kernel<<<1, 1, 0, ctx->stream>>>(r);
            BSN_TRY(launch_check(ctx, "coupled_advance_kernel"));
            if (diag_out)   // the driver's diagnostics of the end-of-step state (BHs after accretion)
                BSN_TRY(diag::launch(ctx, U, nx, ny, nz, dx, dx, dx, x0, y0, z0, r->bh, &r->nbh, nbh, gamma, dpart,
                                     diag_out, &r->t, &r->dt, &r->steps, &r->done, diag_cap, r->led_tot));
            return BSN_OK;
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
        S->U = U; S->nx = nx; S->ny = ny; S->nz = nz; S->nbh = nbh; S->prec = precision; S->variant = variant;
        S->sg = self_gravity; S->torque_free = torque_free; S->evolve = evolve_orbit; S->dx = dx; S->x0 = x0;
        S->y0 = y0; S->z0 = z0; S->gamma = gamma; S->cfl = cfl; S->dt_max = dt_max; S->f_sink = f_sink;
        S->rho_floor = rho_floor; S->P_floor = P_floor; S->t_on = t_bh2_sink_on; S->rho_min = rho_sink_min;
        S->t_end = t_end;
        S->diag_cap = diag_cap;
        memcpy(S->ptrs, ptrs, sizeof(ptrs));
        return BSN_OK;
    };
    if (!same) BSN_TRY(capture());
    const bool settle = n_steps >= 2 && !tile_settled(ctx, TUNE_COUPLED, precision);
    BSN_TRY(graph_replay(ctx, S->exec, S->kernels, settle ? 1 : n_steps, t_end > 0.0, &r->done, S->ev,
                         (volatile int*)((char*)h + sizeof(Dev))));
    if (settle) {   // the tile re-timed on the state after the first step
        BSN_TRY(tile_retime(ctx, TUNE_COUPLED, precision, tune));
        if (tile_code(ctx, precision, base) != variant) {
            variant = tile_code(ctx, precision, base);
            BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            BSN_TRY(capture());
        }
        BSN_TRY(graph_replay(ctx, S->exec, S->kernels, n_steps - 1, t_end > 0.0, &r->done, S->ev,
                             (volatile int*)((char*)h + sizeof(Dev))));
    }
    BSN_CUDA(ctx, cudaMemcpyAsync(h, r, sizeof(Dev), cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    Dev d;
    memcpy(&d, h, sizeof(Dev));
    *t_inout = d.t;
    if (steps_done) *steps_done = d.steps;
    for (int i = 0; i < nbh; ++i) bhs[i] = d.bh[i];
    if (d.done == 2)
        return set_err(ctx, BSN_ERR_NONFINITE, "time step collapsed to 0 at t = %.17g (infinite signal speed)", d.t);
    return BSN_OK;
}

// ---------------------------------------------------------------------------
// The coupled driver loop on nested FMR levels (up to 4).  The reference runs
// coupled_step! on one uniform grid; on nested levels each step is
//   dt = min over levels of the nested CFL (capped by dt_max, clamped to t_end);
//   gas force on every BH from the composite grid (each level's cells except
//   those its child covers); the BH orbit over dt (nbody_step!, FP64);
//   one nested step (fmr3d_step! generalised, fmr_nlevel.cu) whose stages on
//   every level carry BH gravity, self-gravity (Phi frozen per level-0 step,
//   src/fmr_gravity.jl) and sinks in the driver's order, the BHs frozen at
//   their post-orbit state for the whole step;
//   accrete! of every active sink from the finest level over dt;
//   the driver's diagnostics of level 0 (which holds the restriction of the
//   finer levels).
// Time control (dt per level, t, done) lives in the nested plan's device
// record and is mirrored into the coupled record read by the orbit,
// source and accretion kernels.

namespace bsn {
namespace crun {

__global__ void nested_sync_kernel(Dev* r, const fmr::NDev* n) {
    r->dt = n->dt[0];
    r->t = n->t;
    r->done = n->done;
    r->steps = n->steps;
}

}  // namespace crun

void coupled_nested_state_free(bsn_ctx* ctx) {
    fmr::nstate_destroy((fmr::NState*)ctx->coupled_nested_state);
    ctx->coupled_nested_state = nullptr;
}

}  // namespace bsn

extern "C" bsn_status bsn_coupled_nested_run_steps(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, bsn_bh* bhs,
                                                   int nbh, double x0, double y0, double z0, double cfl,
                                                   double dt_max, double f_sink, int torque_free, int self_gravity,
                                                   double t_bh2_sink_on, double rho_sink_min, int evolve_orbit,
                                                   int precision, int n_steps, double t_end, double* t_inout,
                                                   int* steps_done, double* diag_out, int diag_cap) {
    using namespace bsn::fmr;
    if (!ctx) return BSN_ERR_ARG;
    if (!t_inout || (nbh > 0 && !bhs)) return set_err(ctx, BSN_ERR_ARG, "null argument");
    if (nbh < 0 || nbh > MAXBH) return set_err(ctx, BSN_ERR_UNSUPPORTED, "at most %d black holes", MAXBH);
    if (n_steps < 0) return set_err(ctx, BSN_ERR_ARG, "n_steps < 0");
    if (diag_out && diag_cap < 0) return set_err(ctx, BSN_ERR_ARG, "diag_cap < 0");
    if (!diag_out) diag_cap = 0;
    if (!ctx->coupled_nested_state) ctx->coupled_nested_state = new NState();
    NState* S = (NState*)ctx->coupled_nested_state;
    NPlan plan;
    BSN_TRY(make_plan(ctx, pairs, npairs, precision, self_gravity, 1.0, 1, S, plan));
    const int nl = plan.nl;
    bsn_status st;
    Dev* r = (Dev*)slot(ctx, SLOT_CRUN, sizeof(Dev), &st); BSN_TRY(st);
    const int blocks = 148 * 4;
    double* part = (double*)slot(ctx, SLOT_CRED, sizeof(double) * 6 * blocks * nl, &st); BSN_TRY(st);
    double* dpart = nullptr;
    if (diag_out) {
        dpart = (double*)slot(ctx, SLOT_DIAGREC, sizeof(double) * 2 * diag::NDIAG * diag::BLOCKS, &st); BSN_TRY(st);
    }
    // level origins: level k+1 starts at the lower face of level k's cell ci_lo
    double ox[NMAXL], oy[NMAXL], oz[NMAXL];
    ox[0] = x0; oy[0] = y0; oz[0] = z0;
    for (int k = 0; k < npairs; ++k) {
        ox[k + 1] = ox[k] + (double)(pairs[k].ci_lo - 1) * pairs[k].dxc;
        oy[k + 1] = oy[k] + (double)(pairs[k].cj_lo - 1) * pairs[k].dyc;
        oz[k + 1] = oz[k] + (double)(pairs[k].ck_lo - 1) * pairs[k].dzc;
    }
    for (int l = 0; l < nl; ++l) {
        f64::StageArgs& a = plan.base[l];
        a.x0 = ox[l]; a.y0 = oy[l]; a.z0 = oz[l];
        if (nbh > 0) { a.use_bh = 1; a.bh_dev = &r->bsrc; a.use_sink = 1; a.sk_dev = &r->ssrc; }
        plan.led_raw[l] = &r->led[l][0][0];
        a.stiff_guard = 1;
        a.tune_class = TUNE_NESTED;
    }
    plan.led_tot = r->led_tot;
    if (self_gravity) {
        const NLevel& v = plan.L[0];
        if (precision == PREC_F64) BSN_TRY(poisson_prepare(ctx, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz));
        else BSN_TRY(poisson_prepare_f32(ctx, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz));
    }
    // BHs to the device through the pinned buffer, then both records initialised
    double* h = (double*)pinned(ctx, sizeof(Dev) + sizeof(NDev) + 128, &st); BSN_TRY(st);
    bsn_bh* hb = (bsn_bh*)h;
    for (int i = 0; i < nbh; ++i) hb[i] = bhs[i];
    bsn_bh* db = (bsn_bh*)part;
    BSN_CUDA(ctx, cudaMemcpyAsync(db, hb, sizeof(bsn_bh) * (nbh > 0 ? nbh : 1), cudaMemcpyHostToDevice, ctx->stream));
    init_kernel<<<1, 1, 0, ctx->stream>>>(r, *t_inout, db, nbh);
    BSN_TRY(launch_check(ctx, "coupled_init_kernel"));
    n_init_kernel<<<1, 1, 0, ctx->stream>>>(plan.d, *t_inout);
    BSN_TRY(launch_check(ctx, "fmrN_init_kernel"));
    // tile choices before any capture (the autotuner launches and times), on
    // stage-1 work with the loop's BH sources (filled again by the step graph)
    int tiles[NMAXL] = {-1, -1, -1, -1};
    auto tune = [&]() -> bsn_status {
        if (nbh > 0) {
            fill_kernel<<<1, 32, 0, ctx->stream>>>(r, f_sink, torque_free, rho_sink_min, t_bh2_sink_on);
            BSN_TRY(launch_check(ctx, "coupled_fill_kernel"));
        }
        for (int l = 0; l < nl; ++l) {
            f64::StageArgs p = plan.base[l];
            p.Uin = plan.L[l].U; p.dt_dev = nullptr; p.done_dev = nullptr; p.use_reg = 0; p.use_bnd = 0; p.Gh = nullptr;
            BSN_TRY(stage_autotune(ctx, precision, p, plan.L[l].A));
        }
        for (int l = 0; l < nl; ++l) tiles[l] = tile_code(ctx, precision, plan.base[l]);
        return BSN_OK;
    };
    BSN_TRY(tune());

    const NLevel& fin = plan.L[nl - 1];
    std::vector<double> extra = {(double)nbh, x0, y0, z0, dt_max, f_sink, (double)torque_free, t_bh2_sink_on,
                                 rho_sink_min, (double)evolve_orbit, (double)diag_cap,
                                 (double)(uintptr_t)r, (double)(uintptr_t)part, (double)(uintptr_t)diag_out,
                                 (double)(uintptr_t)dpart};
    bool same = S->exec && (int)S->key_pairs.size() == npairs &&
                memcmp(S->key_pairs.data(), pairs, sizeof(bsn_fmr2) * npairs) == 0 && S->prec == precision &&
                S->sg == self_gravity && S->cfl == cfl && S->t_end == t_end &&
                memcmp(S->tiles, tiles, sizeof(tiles)) == 0 && S->key_base == S->arena.base && S->key_extra == extra;
    auto capture = [&]() -> bsn_status {
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
            for (int l = 0; l < nl; ++l) {
                const NLevel& v = plan.L[l];
                BSN_TRY(f64_cfl_fold(ctx, v.U, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz, plan.gamma, &plan.d->sm[l],
                                     &plan.d->nan[l]));
            }
            n_dt_kernel<<<1, 1, 0, ctx->stream>>>(plan.d, cfl, plan.R, t_end, dt_max);
            BSN_TRY(launch_check(ctx, "fmrN_dt_kernel"));
            nested_sync_kernel<<<1, 1, 0, ctx->stream>>>(r, plan.d);
            BSN_TRY(launch_check(ctx, "coupled_nested_sync_kernel"));
            // gas force on every BH from the composite of the levels
            for (int i = 0; i < nbh; ++i) {
                for (int l = 0; l < nl; ++l) {
                    const NLevel& v = plan.L[l];
                    Box skip{{1, 1, 1}, {0, 0, 0}};
                    if (l < nl - 1)
                        for (int d = 0; d < 3; ++d) {
                            skip.lo[d] = plan.P[l].G.lo[d] - 1;
                            skip.hi[d] = plan.P[l].G.hi[d] - 1;
                        }
                    gas_force_kernel<<<blocks, 256, 0, ctx->stream>>>(v.U, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz, ox[l],
                                                                      oy[l], oz[l], r, i, part + 6 * blocks * l, skip);
                    BSN_TRY(launch_check(ctx, "coupled_gas_force_kernel"));
                }
                gas_force_finish<<<1, 256, 0, ctx->stream>>>(part, blocks * nl, r, i);
                BSN_TRY(launch_check(ctx, "coupled_gas_force_finish"));
            }
            if (evolve_orbit && nbh > 0) {
                nbody_kernel<<<1, 32, 0, ctx->stream>>>(r);
                BSN_TRY(launch_check(ctx, "coupled_nbody_kernel"));
            }
            fill_kernel<<<1, 32, 0, ctx->stream>>>(r, f_sink, torque_free, rho_sink_min, t_bh2_sink_on);
            BSN_TRY(launch_check(ctx, "coupled_fill_kernel"));
            BSN_TRY(plan.step());
            for (int i = 0; i < nbh; ++i) {
                accrete_kernel<<<1, 256, 0, ctx->stream>>>(fin.U, fin.nx, fin.ny, fin.nz, fin.dx, fin.dy, fin.dz,
                                                          ox[nl - 1], oy[nl - 1], oz[nl - 1], r, i, f_sink,
                                                          rho_sink_min);
                BSN_TRY(launch_check(ctx, "coupled_accrete_kernel"));
            }
            n_advance_kernel<<<1, 1, 0, ctx->stream>>>(plan.d);
            BSN_TRY(launch_check(ctx, "fmrN_advance_kernel"));
            nested_sync_kernel<<<1, 1, 0, ctx->stream>>>(r, plan.d);
            BSN_TRY(launch_check(ctx, "coupled_nested_sync_kernel"));
            if (diag_out) {
                const NLevel& v = plan.L[0];
                BSN_TRY(diag::launch(ctx, v.U, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz, x0, y0, z0, r->bh, &r->nbh, nbh,
                                     plan.gamma, dpart, diag_out, &r->t, &r->dt, &r->steps, &r->done, diag_cap,
                                     r->led_tot));
            }
            return BSN_OK;
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
        S->key_pairs.assign(pairs, pairs + npairs);
        S->prec = precision; S->sg = self_gravity; S->G_grav = 1.0; S->cfl = cfl; S->t_end = t_end;
        memcpy(S->tiles, tiles, sizeof(tiles));
        S->key_base = S->arena.base;
        S->key_extra = extra;
        return BSN_OK;
    };
    if (!same) BSN_TRY(capture());
    const bool settle = n_steps >= 2 && !tile_settled(ctx, TUNE_NESTED, precision);
    BSN_TRY(graph_replay(ctx, S->exec, S->kernels, settle ? 1 : n_steps, t_end > 0.0, plan.done, S->ev,
                         (volatile int*)((char*)h + sizeof(Dev) + sizeof(NDev))));
    if (settle) {   // the tiles re-timed on the state after the first step
        BSN_TRY(tile_retime(ctx, TUNE_NESTED, precision, tune));
        if (memcmp(S->tiles, tiles, sizeof(tiles)) != 0) {
            BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            BSN_TRY(capture());
        }
        BSN_TRY(graph_replay(ctx, S->exec, S->kernels, n_steps - 1, t_end > 0.0, plan.done, S->ev,
                             (volatile int*)((char*)h + sizeof(Dev) + sizeof(NDev))));
    }
    NDev* hn = (NDev*)((char*)h + sizeof(Dev));
    BSN_CUDA(ctx, cudaMemcpyAsync(h, r, sizeof(Dev), cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaMemcpyAsync(hn, plan.d, sizeof(NDev), cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    Dev d;
    memcpy(&d, h, sizeof(Dev));
    *t_inout = hn->t;
    if (steps_done) *steps_done = hn->steps;
    for (int i = 0; i < nbh; ++i) bhs[i] = d.bh[i];
    if (hn->done == 2)
        return set_err(ctx, BSN_ERR_NONFINITE, "time step collapsed to 0 at t = %.17g (infinite signal speed)", hn->t);
    return BSN_OK;
}
