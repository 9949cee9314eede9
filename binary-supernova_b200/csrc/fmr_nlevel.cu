// fmr_nlevel.cu -- nested fixed mesh refinement with N <= 4 levels (FP64
// parity path; the device time loop also runs the FP32 and learned stencils).
//
// The reference's fmr3d_step! (src/fmr3d.jl:451-604) couples two levels.  Its
// recursive generalisation: a substep of level l runs its SSP-RK3 (ghosts from
// the parent's state interpolated in time for l > 0, flux registers toward its
// child, boundary fluxes into the parent's fine registers), then `ratio`
// substeps of its child with ghosts from (1 - a) U_l^n + a U_l^{n+1},
// a = s / ratio, then restriction, Berger-Colella correction and floors.
// With self-gravity the density is restricted up the chain, Poisson is solved
// once on level 0 and Phi goes down the chain trilinearly, frozen for the step
// (src/fmr_gravity.jl:40-181 applied pair by pair).
//
// Batching: a level's first substep takes its ghosts from the parent at a = 0,
// i.e. from the parent's state at the start of the parent's substep.  So the
// first substeps of a whole chain of levels l, l+1, ..., N-1 are independent
// of each other and each of their three RK3 stages is one persistent launch
// over the blocks of all those levels (stage_kernel_batch).  The remaining
// substeps unwind deepest level first, each again batching its own chain.
// For three levels of ratio 2 that is 6 stage launches per coarse step in place
// of 21.
#include "fmr_nested.cuh"
#include "poisson.cuh"

namespace bsn {
namespace fmr {

__device__ void n_set_level_dts(NDev* d, double dt0, const Ratios& R) {
    d->dt[0] = dt0;
    for (int l = 1; l < R.n; ++l) d->dt[l] = d->dt[l - 1] / (double)R.r[l - 1];
    for (int i = 0; i < NMAXQ; ++i) d->queue[i] = 0u;
}

__global__ void n_init_kernel(NDev* d, double t) {
    for (int l = 0; l < NMAXL; ++l) { d->dt[l] = 0.0; d->sm[l] = 0ull; d->nan[l] = 0u; }
    d->t = t;
    d->done = 0;
    d->steps = 0;
    for (int i = 0; i < NMAXQ; ++i) d->queue[i] = 0u;
}

// one step of a given dt (the host-driven step)
__global__ void n_fixed_dt_kernel(NDev* d, double dt0, Ratios R) { n_set_level_dts(d, dt0, R); }

// cfl_dt_fmr3d over N levels: min over levels of (product of the ratios
// above the level) x cfl / max speed (Inf for a NaN or zero maximum), then the
// dt_max cap (> 0) and the t_end clamp (src/fmr3d.jl:616-622).
__global__ void n_dt_kernel(NDev* d, double cfl, Ratios R, double t_end, double dt_max) {
    if (d->done) return;
    double dt = 0.0;
    int fac = 1;
    for (int l = 0; l < R.n; ++l) {
        double sm = __longlong_as_double((long long)d->sm[l]);
        double dtl = d->nan[l] ? INFINITY : (sm > 0.0 ? cfl / sm : INFINITY);
        if (l == 0) dt = dtl;
        else { fac *= R.r[l - 1]; dt = jmin(dt, (double)fac * dtl); }
        d->sm[l] = 0ull;
        d->nan[l] = 0u;
    }
    if (dt_max > 0.0) dt = jmin(dt, dt_max);
    if (t_end > 0.0) {
        if (!(d->t < t_end)) { d->done = 1; return; }
        dt = jmin(dt, t_end - d->t);
    }
    if (!(dt > 0.0)) { d->done = 2; return; }
    n_set_level_dts(d, dt, R);
}

__global__ void n_advance_kernel(NDev* d) {
    if (d->done) return;
    d->t += d->dt[0];
    d->steps += 1;
}

const double kRkW[3] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};

LedBox NPlan::covered(int l) const {
    LedBox b;
    if (l < nl - 1)
        for (int d = 0; d < 3; ++d) {
            b.lo[d] = P[l].G.lo[d] - 1;
            b.hi[d] = P[l].G.hi[d];
        }
    return b;
}

bsn_status NPlan::chain(int l, double alpha) {
    // substep starts of levels l..nl-1: saved states and fresh registers
    for (int k = l; k < nl - 1; ++k) {
        long long n = Geom(L[k].nx, L[k].ny, L[k].nz).nelem();
        copy_kernel<<<grid1d(std::min<long long>(n, 148LL * 8 * 256), 256), 256, 0, ctx->stream>>>(L[k].Ucn, L[k].U,
                                                                                                     n, done);
        BSN_TRY(launch_check(ctx, "fmr_copy_kernel"));
        zero_kernel<<<grid1d(std::min<long long>(P[k].nregs, 148LL * 8 * 256), 256), 256, 0, ctx->stream>>>(
            P[k].regs, P[k].nregs, done);
        BSN_TRY(launch_check(ctx, "fmr_zero_kernel"));
    }
    if (l > 0) BSN_TRY(prolong_ghosts(ctx, P[l - 1].G, L[l - 1].Ucn, L[l - 1].U, alpha, L[l].Gh, done));
    for (int k = l + 1; k < nl; ++k)
        BSN_TRY(prolong_ghosts(ctx, P[k - 1].G, L[k - 1].Ucn, nullptr, 0.0, L[k].Gh, done));
    for (int s = 0; s < 3; ++s) {
        const int nb = nl - l;
        f64::StageBatch B;
        memset(&B, 0, sizeof(B));
        B.nlev = nb;
        for (int k = l; k < nl; ++k) {
            f64::StageArgs& a = B.lv[k - l];
            a = base[k];
            double* in[3] = {L[k].U, L[k].A, L[k].B};
            double* out[3] = {L[k].A, L[k].B, L[k].U};
            a.Uin = in[s]; a.Un = L[k].U; a.Uout = out[s];
            set_stage(a, s + 1, 0.0);
            a.reg.wt = kRkW[s];
            if (led_raw[k]) {
                a.ledger = led_raw[k] + f64::LED_TERMS * s;
                a.led_bnd = k == 0;
                const LedBox cv = covered(k);
                for (int d = 0; d < 3; ++d) { a.led_skip_lo[d] = cv.lo[d]; a.led_skip_hi[d] = cv.hi[d]; }
            }
        }
        if (nb == 1) {
            BSN_TRY(stage_launch(ctx, prec, B.lv[0]));
        } else {
            if (qn >= NMAXQ) return set_err(ctx, BSN_ERR_UNSUPPORTED, "more than %d batched launches per step", NMAXQ);
            B.queue = &d->queue[qn++];
            BSN_TRY(stage_launch_batch(ctx, prec, B));
        }
        for (int k = std::max(l, 1); k < nl; ++k) {
            const NPair& p = P[k - 1];
            const double rr = (double)(p.G.r * p.G.r);
            fine_reg_kernel<<<grid1d(p.nfine, 128), 128, 0, ctx->stream>>>(p.G, p.Rf, 0.0, &d->dt[k], kRkW[s], rr,
                                                                             done);
            BSN_TRY(launch_check(ctx, "fine_reg_kernel"));
        }
    }
    for (int k = l; k < nl; ++k)
        if (led_raw[k]) BSN_TRY(f64_ledger_fold(ctx, led_raw[k], led_tot, &d->dt[k], done));
    for (int k = l; k < nl; ++k)
        BSN_TRY(f64_ghost_combine(ctx, L[k].U, k == 0 ? L[0].B : nullptr, k == 0 ? nullptr : L[k].Gh, L[k].nx,
                                  L[k].ny, L[k].nz, bc, 0.0, &d->dt[k], done));
    // unwind: the remaining substeps of each child, deepest first, then
    // restriction, Berger-Colella correction and floors of the parent
    for (int k = nl - 2; k >= l; --k) {
        const int r = P[k].G.r;
        for (int sub = 1; sub < r; ++sub) BSN_TRY(chain(k + 1, (double)sub / (double)r));
        BSN_TRY(restrict_(ctx, P[k].G, L[k].U, L[k + 1].U, 5, done));
        bc_correct_kernel<<<grid1d(P[k].ncorr, 128), 128, 0, ctx->stream>>>(
            P[k].G, P[k].Rc, P[k].Rf, L[k].U, 1.0 / L[k].dx, 1.0 / L[k].dy, 1.0 / L[k].dz, done);
        BSN_TRY(launch_check(ctx, "bc_correct_kernel"));
        BSN_TRY(f64_floors(ctx, L[k].U, L[k].nx, L[k].ny, L[k].nz, rho_floor, P_floor, gamma, done,
                           led_tot ? led_tot + f64::LEDT_FLOORS : nullptr, covered(k),
                           L[k].dx * L[k].dy * L[k].dz));
    }
    return BSN_OK;
}

// density restricted up the chain (deepest pair first), one isolated solve on
// level 0, trilinear Phi down the chain, then the G scaling on every level
bsn_status NPlan::gravity() {
    for (int k = nl - 2; k >= 0; --k) BSN_TRY(restrict_(ctx, P[k].G, L[k].U, L[k + 1].U, 1, done));
    if (prec == PREC_F64)
        BSN_TRY(poisson_from_state(ctx, L[0].U, L[0].nx, L[0].ny, L[0].nz, L[0].dx, L[0].dy, L[0].dz, -1.0, L[0].phi));
    else
        BSN_TRY(poisson_from_state_f32(ctx, L[0].U, L[0].nx, L[0].ny, L[0].nz, L[0].dx, L[0].dy, L[0].dz, -1.0,
                                       L[0].phi));
    for (int k = 0; k < nl - 1; ++k) {
        long long n = (long long)L[k + 1].nx * L[k + 1].ny * L[k + 1].nz;
        trilinear_kernel<<<grid1d(n, 256), 256, 0, ctx->stream>>>(P[k].G, L[k].phi, L[k + 1].phi);
        BSN_TRY(launch_check(ctx, "trilinear_kernel"));
    }
    if (G_grav != 1.0)
        for (int k = 0; k < nl; ++k) {
            long long n = (long long)L[k].nx * L[k].ny * L[k].nz;
            scale_kernel<<<grid1d(n, 256), 256, 0, ctx->stream>>>(L[k].phi, n, G_grav);
            BSN_TRY(launch_check(ctx, "scale_kernel"));
        }
    return BSN_OK;
}

bsn_status NPlan::step() {
    qn = 0;
    if (sg) BSN_TRY(gravity());
    return chain(0, 0.0);
}

static size_t align_up(size_t b) { return (b + 255) & ~(size_t)255; }

// Validate the chain, lay out the arena and fill the plan.
bsn_status make_plan(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, int prec, int sg, double G_grav, int guard,
                            NState* S, NPlan& plan) {
    if (!pairs || npairs < 1 || npairs > NMAXL - 1)
        return set_err(ctx, BSN_ERR_ARG, "need 1..%d level pairs, got %d", NMAXL - 1, npairs);
    if (prec != PREC_F64 && prec != PREC_F32 && prec != PREC_LEARNED)
        return set_err(ctx, BSN_ERR_ARG, "bad precision %d", prec);
    plan.ctx = ctx;
    plan.nl = npairs + 1;
    plan.prec = prec;
    plan.sg = sg;
    plan.G_grav = G_grav;
    plan.gamma = pairs[0].gamma;
    plan.bc = pairs[0].bc;
    plan.rho_floor = pairs[0].rho_floor;
    plan.P_floor = pairs[0].P_floor;
    plan.R.n = plan.nl;
    for (int k = 0; k < npairs; ++k) {
        BSN_TRY(make_geo(ctx, &pairs[k], plan.P[k].G));
        plan.R.r[k] = pairs[k].ratio;
        if (k + 1 < npairs) {
            const bsn_fmr2 &a = pairs[k], &b = pairs[k + 1];
            if (a.Uf != b.Uc || a.nfx != b.ncx || a.nfy != b.ncy || a.nfz != b.ncz || a.dxf != b.dxc ||
                a.dyf != b.dyc || a.dzf != b.dzc)
                return set_err(ctx, BSN_ERR_ARG, "level pair %d's fine level is not pair %d's coarse level", k, k + 1);
        }
    }
    for (int l = 0; l < plan.nl; ++l) {
        NLevel& v = plan.L[l];
        if (l < npairs) {
            v.U = pairs[l].Uc; v.nx = pairs[l].ncx; v.ny = pairs[l].ncy; v.nz = pairs[l].ncz;
            v.dx = pairs[l].dxc; v.dy = pairs[l].dyc; v.dz = pairs[l].dzc;
        } else {
            const bsn_fmr2& p = pairs[npairs - 1];
            v.U = p.Uf; v.nx = p.nfx; v.ny = p.nfy; v.nz = p.nfz; v.dx = p.dxf; v.dy = p.dyf; v.dz = p.dzf;
        }
        BSN_TRY(check_dims(ctx, v.nx, v.ny, v.nz));
    }
    // arena layout
    size_t off = align_up(sizeof(NDev));
    size_t lo_[NMAXL][5];
    for (int l = 0; l < plan.nl; ++l) {
        size_t ne = sizeof(double) * (size_t)Geom(plan.L[l].nx, plan.L[l].ny, plan.L[l].nz).nelem();
        size_t na = sizeof(double) * (size_t)plan.L[l].nx * plan.L[l].ny * plan.L[l].nz;
        lo_[l][0] = off; off += align_up(ne);                               // A
        lo_[l][1] = off; off += align_up(ne);                               // B
        lo_[l][2] = off; off += l < plan.nl - 1 ? align_up(ne) : 0;         // Ucn
        lo_[l][3] = off; off += l > 0 ? align_up(ne) : 0;                   // Gh
        lo_[l][4] = off; off += sg ? align_up(na) : 0;                      // phi
    }
    size_t po[NMAXL - 1][2];
    for (int k = 0; k < npairs; ++k) {
        const Geo& G = plan.P[k].G;
        long long nic = G.hi[0] - G.lo[0] + 1, njc = G.hi[1] - G.lo[1] + 1, nkc = G.hi[2] - G.lo[2] + 1;
        long long e3 = 5 * (njc * nkc + nic * nkc + nic * njc);
        plan.P[k].nregs = 4 * e3;
        plan.P[k].nfine = 2 * e3;
        plan.P[k].ncorr = e3;
        po[k][0] = off; off += align_up(sizeof(double) * (size_t)plan.P[k].nregs);
        long long ef = 2LL * 5 * ((long long)G.nfy * G.nfz + (long long)G.nfx * G.nfz + (long long)G.nfx * G.nfy);
        po[k][1] = off; off += align_up(sizeof(double) * (size_t)ef);
    }
    if (S->arena.bytes < off) {
        if (S->arena.base) {
            BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            S->release();
            cudaFree(S->arena.base);
            S->arena.base = nullptr;
            S->arena.bytes = 0;
        }
        BSN_CUDA(ctx, cudaMalloc(&S->arena.base, off));
        S->arena.bytes = off;
    }
    char* b = (char*)S->arena.base;
    plan.d = (NDev*)b;
    plan.done = &plan.d->done;
    for (int l = 0; l < plan.nl; ++l) {
        NLevel& v = plan.L[l];
        v.A = (double*)(b + lo_[l][0]);
        v.B = (double*)(b + lo_[l][1]);
        v.Ucn = l < plan.nl - 1 ? (double*)(b + lo_[l][2]) : nullptr;
        v.Gh = l > 0 ? (double*)(b + lo_[l][3]) : nullptr;
        v.phi = sg ? (double*)(b + lo_[l][4]) : nullptr;
    }
    for (int k = 0; k < npairs; ++k) {
        NPair& p = plan.P[k];
        const Geo& G = p.G;
        long long nic = G.hi[0] - G.lo[0] + 1, njc = G.hi[1] - G.lo[1] + 1, nkc = G.hi[2] - G.lo[2] + 1;
        long long e[3] = {5 * njc * nkc, 5 * nic * nkc, 5 * nic * njc};
        p.regs = (double*)(b + po[k][0]);
        double* q = p.regs;
        for (int D = 0; D < 3; ++D) for (int s = 0; s < 2; ++s) { p.Rc.r[2 * D + s] = q; q += e[D]; }
        for (int D = 0; D < 3; ++D) for (int s = 0; s < 2; ++s) { p.Rf.r[2 * D + s] = q; q += e[D]; }
        long long ef[3] = {5LL * G.nfy * G.nfz, 5LL * G.nfx * G.nfz, 5LL * G.nfx * G.nfy};
        double* bf = (double*)(b + po[k][1]);
        for (int D = 0; D < 3; ++D) for (int s = 0; s < 2; ++s) { p.Rf.bnd[2 * D + s] = bf; bf += ef[D]; }
        for (int i = 0; i < 6; ++i) p.Rc.bnd[i] = nullptr;
    }
    // stage arguments per level: registers toward the child, boundary faces
    // toward the parent, ghosts from the parent's interpolation
    for (int l = 0; l < plan.nl; ++l) {
        f64::StageArgs& a = plan.base[l];
        const NLevel& v = plan.L[l];
        stage_args_init(a, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz, plan.gamma, plan.bc, plan.rho_floor, plan.P_floor);
        a.stiff_guard = guard;   // FP32 faces of stiff stencils in FP64 (sinks beside dense gas)
        if (l < plan.nl - 1) {
            const Geo& G = plan.P[l].G;
            a.use_reg = 1;
            for (int i = 0; i < 6; ++i) a.reg.reg[i] = plan.P[l].Rc.r[i];
            for (int D = 0; D < 3; ++D) {
                a.reg.lo[D] = G.lo[D] - 1;
                a.reg.hi[D] = G.hi[D];
                a.reg.t0[D] = G.lo[D] - 1;
                a.reg.t1[D] = G.hi[D] - 1;
            }
        }
        if (l > 0) {
            a.Gh = v.Gh;
            a.use_bnd = 1;
            for (int i = 0; i < 6; ++i) a.bnd.f[i] = const_cast<double*>(plan.P[l - 1].Rf.bnd[i]);
        }
        if (sg) { a.use_sg = 1; a.phi = v.phi; }
        a.dt_dev = &plan.d->dt[l];
        a.done_dev = plan.done;
    }
    return BSN_OK;
}

static NState* nstate(bsn_ctx* ctx) {
    if (!ctx->fmrN_state) ctx->fmrN_state = new NState();
    return (NState*)ctx->fmrN_state;
}

// One nested step of a given dt0 (host-driven; FP64).
bsn_status fmrN_step(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, double dt0, int sg, double G_grav) {
    NState* S = nstate(ctx);
    NPlan plan;
    BSN_TRY(make_plan(ctx, pairs, npairs, PREC_F64, sg, G_grav, ctx->stiff_guard, S, plan));
    n_init_kernel<<<1, 1, 0, ctx->stream>>>(plan.d, 0.0);
    BSN_TRY(launch_check(ctx, "fmrN_init_kernel"));
    n_fixed_dt_kernel<<<1, 1, 0, ctx->stream>>>(plan.d, dt0, plan.R);
    BSN_TRY(launch_check(ctx, "fmrN_dt_kernel"));
    return plan.step();
}

bsn_status fmrN_cfl(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, double cfl, double* dt_out) {
    if (!pairs || npairs < 1 || npairs > NMAXL - 1)
        return set_err(ctx, BSN_ERR_ARG, "need 1..%d level pairs, got %d", NMAXL - 1, npairs);
    const bsn_fmr2& p0 = pairs[0];
    double dt;
    BSN_TRY(f64_cfl_dt(ctx, p0.Uc, p0.ncx, p0.ncy, p0.ncz, p0.dxc, p0.dyc, p0.dzc, p0.gamma, cfl, &dt));
    int fac = 1;
    for (int k = 0; k < npairs; ++k) {
        const bsn_fmr2& p = pairs[k];
        double dtk;
        BSN_TRY(f64_cfl_dt(ctx, p.Uf, p.nfx, p.nfy, p.nfz, p.dxf, p.dyf, p.dzf, p0.gamma, cfl, &dtk));
        fac *= p.ratio;
        dt = jmin(dt, (double)fac * dtk);
    }
    *dt_out = dt;
    return BSN_OK;
}

// The driver loop `dt = cfl_dt(levels); dt = min(dt, t_end - t); step; t += dt`
// on the device, one CUDA graph per coarse step.
bsn_status fmrN_run(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, double cfl, int prec, int sg, double G_grav,
                    int n_steps, double t_end, double* t_inout, int* steps_done) {
    if (n_steps < 0 || !t_inout) return set_err(ctx, BSN_ERR_ARG, "bad n_steps or null t_inout");
    NState* S = nstate(ctx);
    NPlan plan;
    BSN_TRY(make_plan(ctx, pairs, npairs, prec, sg, G_grav, ctx->stiff_guard, S, plan));
    if (sg) {
        const NLevel& v = plan.L[0];
        if (prec == PREC_F64) BSN_TRY(poisson_prepare(ctx, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz));
        else BSN_TRY(poisson_prepare_f32(ctx, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz));
    }
    // tile choices before any capture (the autotuner launches and times)
    int tiles[NMAXL] = {-1, -1, -1, -1};
    for (int l = 0; l < plan.nl; ++l) plan.base[l].tune_class = TUNE_FMR_N;
    auto tune = [&]() -> bsn_status {
        for (int l = 0; l < plan.nl; ++l) {
            f64::StageArgs p = plan.base[l];
            p.Uin = plan.L[l].U; p.dt_dev = nullptr; p.done_dev = nullptr; p.use_reg = 0; p.use_bnd = 0; p.Gh = nullptr;
            BSN_TRY(stage_autotune(ctx, prec, p, plan.L[l].A));
        }
        for (int l = 0; l < plan.nl; ++l) tiles[l] = tile_code(ctx, prec, plan.base[l]);
        return BSN_OK;
    };
    BSN_TRY(tune());
    n_init_kernel<<<1, 1, 0, ctx->stream>>>(plan.d, *t_inout);
    BSN_TRY(launch_check(ctx, "fmrN_init_kernel"));

    bool same = S->exec && (int)S->key_pairs.size() == npairs &&
                memcmp(S->key_pairs.data(), pairs, sizeof(bsn_fmr2) * npairs) == 0 && S->prec == prec &&
                S->sg == sg && S->G_grav == G_grav && S->cfl == cfl && S->t_end == t_end &&
                memcmp(S->tiles, tiles, sizeof(tiles)) == 0 && S->key_base == S->arena.base;
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
            for (int l = 0; l < plan.nl; ++l) {
                const NLevel& v = plan.L[l];
                BSN_TRY(f64_cfl_fold(ctx, v.U, v.nx, v.ny, v.nz, v.dx, v.dy, v.dz, plan.gamma, &plan.d->sm[l],
                                     &plan.d->nan[l]));
            }
            n_dt_kernel<<<1, 1, 0, ctx->stream>>>(plan.d, cfl, plan.R, t_end, 0.0);
            BSN_TRY(launch_check(ctx, "fmrN_dt_kernel"));
            BSN_TRY(plan.step());
            n_advance_kernel<<<1, 1, 0, ctx->stream>>>(plan.d);
            return launch_check(ctx, "fmrN_advance_kernel");
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
        S->prec = prec; S->sg = sg; S->G_grav = G_grav; S->cfl = cfl; S->t_end = t_end;
        memcpy(S->tiles, tiles, sizeof(tiles));
        S->key_base = S->arena.base;
        return BSN_OK;
    };
    if (!same) BSN_TRY(capture());
    bsn_status st;
    double* h = (double*)pinned(ctx, 128 + sizeof(NDev), &st); BSN_TRY(st);
    const bool settle = n_steps >= 2 && !tile_settled(ctx, TUNE_FMR_N, prec);
    BSN_TRY(graph_replay(ctx, S->exec, S->kernels, settle ? 1 : n_steps, t_end > 0.0, plan.done, S->ev,
                         (volatile int*)(h + 8)));
    if (settle) {   // the tiles re-timed on the state after the first step
        BSN_TRY(tile_retime(ctx, TUNE_FMR_N, prec, tune));
        if (memcmp(S->tiles, tiles, sizeof(tiles)) != 0) {
            BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            BSN_TRY(capture());
        }
        BSN_TRY(graph_replay(ctx, S->exec, S->kernels, n_steps - 1, t_end > 0.0, plan.done, S->ev,
                             (volatile int*)(h + 8)));
    }
    NDev* hd = (NDev*)(h + 16);
    BSN_CUDA(ctx, cudaMemcpyAsync(hd, plan.d, sizeof(NDev), cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *t_inout = hd->t;
    if (steps_done) *steps_done = hd->steps;
    if (hd->done == 2)
        return set_err(ctx, BSN_ERR_NONFINITE, "time step collapsed to 0 at t = %.17g (infinite signal speed)", hd->t);
    return BSN_OK;
}

}  // namespace fmr

namespace fmr {
void nstate_destroy(NState* S) {
    if (!S) return;
    S->release();
    if (S->arena.base) cudaFree(S->arena.base);
    if (S->cap) cudaStreamDestroy(S->cap);
    for (cudaEvent_t e : S->ev)
        if (e) cudaEventDestroy(e);
    delete S;
}
}  // namespace fmr

void fmrN_state_free(bsn_ctx* ctx) {
    fmr::nstate_destroy((fmr::NState*)ctx->fmrN_state);
    ctx->fmrN_state = nullptr;
}

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_fmr_nested_step_f64(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, double dt0,
                                        int self_gravity, double G_grav) {
    if (!ctx) return BSN_ERR_ARG;
    return fmr::fmrN_step(ctx, pairs, npairs, dt0, self_gravity, G_grav);
}

extern "C" bsn_status bsn_cfl_dt_fmr_nested_f64(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, double cfl,
                                          double* dt_out) {
    if (!ctx) return BSN_ERR_ARG;
    if (!dt_out) return set_err(ctx, BSN_ERR_ARG, "dt_out is null");
    return fmr::fmrN_cfl(ctx, pairs, npairs, cfl, dt_out);
}

extern "C" bsn_status bsn_fmr_nested_run_steps(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, double cfl, int precision,
                                         int self_gravity, double G_grav, int n_steps, double t_end,
                                         double* t_inout, int* steps_done) {
    if (!ctx) return BSN_ERR_ARG;
    return fmr::fmrN_run(ctx, pairs, npairs, cfl, precision, self_gravity, G_grav, n_steps, t_end, t_inout,
                         steps_done);
}
