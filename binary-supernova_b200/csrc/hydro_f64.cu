// hydro_f64.cu -- FP64 (parity) uniform-grid path: ghost fill, floors, the
// fused RK3 stage, euler3d_rhs!, euler3d_step!, cfl_dt_3d.
// Compiled with -fmad=false: bit-identical to the reference's CPU arithmetic.
#include "hydro_f64.cuh"
#include "stage_launch.cuh"
#include "stage_tile.cuh"

namespace bsn {
namespace f64 {

// ---------------------------------------------------------------------------
// Ghost cells of the whole ghosted array, enumerated slab by slab:
// z-ghost planes (full x,y), y-ghost rows (full x, active z), x-ghost cells
// (active y,z).  Every ghost copies the composed boundary source cell
// (x -> y -> z fill order of src/euler3d.jl:33-62).
struct GhostEnum {
    int nx, ny, nz;
    long long nzg, nyg, nxg;   // counts of each slab family
    __host__ __device__ GhostEnum(int a, int b, int c) : nx(a), ny(b), nz(c) {
        long long X = a + 2 * BSN_NG, Y = b + 2 * BSN_NG;
        nzg = 2LL * BSN_NG * X * Y;
        nyg = 2LL * BSN_NG * X * c;
        nxg = 2LL * BSN_NG * b * c;
    }
    __host__ __device__ long long total() const { return nzg + nyg + nxg; }
    // ghosted 0-based coordinates of ghost number t
    __device__ void coords(long long t, int& i, int& j, int& k) const {
        int X = nx + 2 * BSN_NG, Y = ny + 2 * BSN_NG;
        if (t < nzg) {
            i = (int)(t % X); long long r = t / X; j = (int)(r % Y); int s = (int)(r / Y);
            k = s < BSN_NG ? s : nz + s;            // 0..2, then nz+3..nz+5
        } else if ((t -= nzg) < nyg) {
            i = (int)(t % X); long long r = t / X; int s = (int)(r % (2 * BSN_NG)); k = (int)(r / (2 * BSN_NG)) + BSN_NG;
            j = s < BSN_NG ? s : ny + s;
        } else {
            t -= nyg;
            int s = (int)(t % (2 * BSN_NG)); long long r = t / (2 * BSN_NG);
            j = (int)(r % ny) + BSN_NG; k = (int)(r / ny) + BSN_NG;
            i = s < BSN_NG ? s : nx + s;
        }
    }
};

__global__ void ghost_fill_kernel(double* U, int nx, int ny, int nz, int bc) {
    GhostEnum E(nx, ny, nz);
    Geom G(nx, ny, nz);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= E.total()) return;
    int i, j, k;
    E.coords(t, i, j, k);
    long long dst = G.at(i, j, k);
    long long src = G.act(bc_map(i - BSN_NG, nx, bc), bc_map(j - BSN_NG, ny, bc), bc_map(k - BSN_NG, nz, bc));
#pragma unroll
    for (int q = 0; q < 5; ++q) U[dst + q] = U[src + q];
}

// Final ghost values of euler3d_step!/coupled_step!: the stage-3 combine over
// ghost cells, where dU = 0 and U holds the ghost fill of the stage-2 state:
// U_g = ((1/3) U_g + (2/3) S_g) + ((2/3) dt) * 0.  S is the stage-2 state
// seen through the boundary map (Gh == null) or an explicit ghost buffer.
__global__ void ghost_combine_kernel(double* U, const double* S, const double* Gh, int nx, int ny, int nz,
                                     int bc, double cz, const double* dt_dev, const int* done_dev) {
    if (done_dev && *done_dev) return;
    if (dt_dev) cz = ((2.0 / 3.0) * *dt_dev) * 0.0;
    GhostEnum E(nx, ny, nz);
    Geom G(nx, ny, nz);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= E.total()) return;
    int i, j, k;
    E.coords(t, i, j, k);
    long long dst = G.at(i, j, k);
    const double* src;
    long long so;
    if (Gh) { src = Gh; so = dst; }
    else {
        src = S;
        so = G.act(bc_map(i - BSN_NG, nx, bc), bc_map(j - BSN_NG, ny, bc), bc_map(k - BSN_NG, nz, bc));
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) U[dst + q] = (1.0 / 3.0) * U[dst + q] + (2.0 / 3.0) * src[so + q] + cz;
}

// led (may be null): the floors' change of rho dV on the cells outside the
// half-open box [lo, hi) is added there (mass ledger).
__global__ void floors_kernel(double* U, int nx, int ny, int nz, double rho_floor, double P_floor, double Pfl_gm1,
                              double gm1, const int* done, double* led = nullptr, LedBox skip = LedBox{},
                              double dV = 0.0) {
    if (done && *done) return;
    Geom G(nx, ny, nz);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = (long long)nx * ny * nz;
    if (t >= n) return;
    int a = (int)(t % nx); long long r = t / nx; int b = (int)(r % ny); int c = (int)(r / ny);
    long long o = G.act(a, b, c);
    double v[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) v[q] = U[o + q];
    const double rho0 = v[0];
    apply_floor(v[0], v[1], v[2], v[3], v[4], rho_floor, P_floor, Pfl_gm1, gm1);
#pragma unroll
    for (int q = 0; q < 5; ++q) U[o + q] = v[q];
    if (led && v[0] != rho0 && !skip.has(a, b, c)) atomicAdd(led, (v[0] - rho0) * dV);
}

// Mass ledger of one SSP-RK3 step (or substep) from its per-stage sums raw[3]
// [LED_TERMS] (stage_tile.cuh): a change to stage s's result reaches the
// step's result with the weight the later combines give it -- the stage-1
// right-hand side and result 0.25 * 2/3, stage 2's 2/3, stage 3's 1 (times
// dt for the right-hand sides, whose stage coefficients are dt, dt/4 and
// 2dt/3) -- and the input floors of stages 2 and 3 the weights of the stage
// results they alter.  Adds into tot[LEDT_*] and clears raw.
__global__ void ledger_fold_kernel(double* raw, double* tot, const double* dt_dev, const int* done) {
    if ((done && *done) || threadIdx.x != 0 || blockIdx.x != 0) return;
    const double dt = *dt_dev, c1 = 0.25 * (2.0 / 3.0), c3 = 2.0 / 3.0;
    double(*r)[f64::LED_TERMS] = reinterpret_cast<double(*)[f64::LED_TERMS]>(raw);
    using namespace f64;
    tot[LEDT_FLOORS] += ((c1 * r[0][LED_POST] + c1 * r[1][LED_PRE]) + (c3 * r[1][LED_POST] + c3 * r[2][LED_PRE])) +
                        r[2][LED_POST];
    tot[LEDT_OUTFLOW] -= dt * ((c1 * r[0][LED_BND] + c1 * r[1][LED_BND]) + c3 * r[2][LED_BND]);
    tot[LEDT_DRAINED] += dt * ((c1 * r[0][LED_DRAIN] + c1 * r[1][LED_DRAIN]) + c3 * r[2][LED_DRAIN]);
    for (int s = 0; s < 3; ++s)
        for (int q = 0; q < LED_TERMS; ++q) r[s][q] = 0.0;
}

// cfl_dt_3d speeds folded into a device max (src/gpu_kernels.jl:174-191).
__global__ void cfl_kernel(const double* U, int nx, int ny, int nz, double g, double gm1, double idx, double idy,
                           double idz, unsigned long long* smax_out, unsigned int* nan_out) {
    Geom G(nx, ny, nz);
    __shared__ double red[32];
    __shared__ unsigned int nanf;
    if (threadIdx.x == 0) nanf = 0;
    __syncthreads();
    long long n = (long long)nx * ny * nz;
    double m = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int a = (int)(t % nx); long long r = t / nx; int b = (int)(r % ny); int c = (int)(r / ny);
        long long o = G.act(a, b, c);
        double s = cfl_speed(U[o], U[o + 1], U[o + 2], U[o + 3], U[o + 4], g, gm1, idx, idy, idz);
        if (s != s) nanf = 1;
        else m = fmax(m, s);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mm = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mm = fmax(mm, red[w]);
        atomicMax(smax_out, (unsigned long long)__double_as_longlong(mm));
        if (nanf) atomicOr(nan_out, 1u);
    }
}

}  // namespace f64

using namespace f64;

bsn_status check_dims(bsn_ctx* ctx, int nx, int ny, int nz) {
    if (!ctx) return BSN_ERR_ARG;
    if (nx < 1 || ny < 1 || nz < 1) return set_err(ctx, BSN_ERR_ARG, "grid sizes must be >= 1 (got %d,%d,%d)", nx, ny, nz);
    if ((long long)(nx + 6) * (ny + 6) * (nz + 6) * 5 > (1LL << 40))
        return set_err(ctx, BSN_ERR_UNSUPPORTED, "grid too large");
    return BSN_OK;
}

bsn_status f64_fill_ghosts(bsn_ctx* ctx, double* U, int nx, int ny, int nz, int bc) {
    GhostEnum E(nx, ny, nz);
    ghost_fill_kernel<<<grid1d(E.total(), 256), 256, 0, ctx->stream>>>(U, nx, ny, nz, bc);
    return launch_check(ctx, "ghost_fill_kernel");
}

bsn_status f64_floors(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double rho_floor, double P_floor, double gamma,
                      const int* done_dev, double* led, LedBox skip, double dV) {
    double gm1 = gamma - 1.0;
    prof_begin(ctx);
    floors_kernel<<<grid1d((long long)nx * ny * nz, 256), 256, 0, ctx->stream>>>(
        U, nx, ny, nz, rho_floor, P_floor, P_floor / gm1, gm1, done_dev, led, skip, dV);
    return launch_check(ctx, "floors_kernel");
}

bsn_status f64_ledger_fold(bsn_ctx* ctx, double* raw, double* tot, const double* dt_dev, const int* done_dev) {
    ledger_fold_kernel<<<1, 32, 0, ctx->stream>>>(raw, tot, dt_dev, done_dev);
    return launch_check(ctx, "ledger_fold_kernel");
}

bsn_status f64_ghost_combine(bsn_ctx* ctx, double* U, const double* S, const double* Gh, int nx, int ny, int nz,
                             int bc, double dt, const double* dt_dev, const int* done_dev) {
    GhostEnum E(nx, ny, nz);
    double cz = ((2.0 / 3.0) * dt) * 0.0;
    prof_begin(ctx);
    ghost_combine_kernel<<<grid1d(E.total(), 256), 256, 0, ctx->stream>>>(U, S, Gh, nx, ny, nz, bc, cz, dt_dev,
                                                                          done_dev);
    return launch_check(ctx, "ghost_combine_kernel");
}

void stage_args_init(StageArgs& A, int nx, int ny, int nz, double dx, double dy, double dz, double gamma, int bc,
                     double rho_floor, double P_floor) {
    memset(&A, 0, sizeof(A));
    A.nx = nx; A.ny = ny; A.nz = nz; A.bc = bc;
    A.g = gamma; A.gm1 = gamma - 1.0;
    A.rho_floor = rho_floor; A.P_floor = P_floor; A.Pfl_gm1 = P_floor / (gamma - 1.0);
    A.idx = 1.0 / dx; A.idy = 1.0 / dy; A.idz = 1.0 / dz;
    A.dx = dx; A.dy = dy; A.dz = dz;
    A.inv2dx = 0.5 / dx; A.inv2dy = 0.5 / dy; A.inv2dz = 0.5 / dz;
}

// FP64 tile variants of the fused stage kernel (bitwise identical results:
// every interface and every cell is computed by the same arithmetic whatever
// the tiling).  MINB keeps two 256-thread CTAs (or the equivalent) per SM.
namespace {
const TileVariant kF64Variants[] = {{8, 8, 8, 256, 2}, {8, 8, 4, 128, 4}, {16, 8, 4, 256, 2}, {16, 8, 8, 512, 1}};

template <int TX, int TY, int TZ, int NT, int MINB>
bsn_status launch_f64(bsn_ctx* ctx, const StageArgs& A) {
    bool tma_used = false;
    BSN_TRY((tile::launch_tma<tile::F64Physics, TX, TY, TZ, NT, MINB>(ctx, A, "stage_kernel_tma", &tma_used)));
    if (tma_used) return BSN_OK;
    return tile::launch_plain<tile::F64Physics, TX, TY, TZ, NT, MINB>(
        ctx, A, tile::smem_bytes<tile::F64Physics, TX, TY, TZ>(), "stage_kernel");
}
}  // namespace

int f64_variant_count() { return (int)(sizeof(kF64Variants) / sizeof(kF64Variants[0])); }
TileVariant f64_variant(int idx) { return kF64Variants[idx]; }
bsn_status f64_launch_variant(bsn_ctx* ctx, int idx, const StageArgs& A) {
    switch (idx) {
        case 0: return launch_f64<8, 8, 8, 256, 2>(ctx, A);
        case 1: return launch_f64<8, 8, 4, 128, 4>(ctx, A);
        case 2: return launch_f64<16, 8, 4, 256, 2>(ctx, A);
        case 3: return launch_f64<16, 8, 8, 512, 1>(ctx, A);
        default: return set_err(ctx, BSN_ERR_ARG, "no FP64 tile variant %d", idx);
    }
}

bsn_status f64_launch_batch_variant(bsn_ctx* ctx, int idx, const StageBatch& B) {
    using P = tile::F64Physics;
    switch (idx) {
        case 0: return tile::launch_batch<P, 8, 8, 8, 256, 2>(ctx, B, tile::smem_bytes<P, 8, 8, 8>(), "stage_kernel_batch");
        case 1: return tile::launch_batch<P, 8, 8, 4, 128, 4>(ctx, B, tile::smem_bytes<P, 8, 8, 4>(), "stage_kernel_batch");
        case 2: return tile::launch_batch<P, 16, 8, 4, 256, 2>(ctx, B, tile::smem_bytes<P, 16, 8, 4>(), "stage_kernel_batch");
        case 3: return tile::launch_batch<P, 16, 8, 8, 512, 1>(ctx, B, tile::smem_bytes<P, 16, 8, 8>(), "stage_kernel_batch");
        default: return set_err(ctx, BSN_ERR_ARG, "no FP64 tile variant %d", idx);
    }
}

bsn_status f64_launch_stage(bsn_ctx* ctx, const StageArgs& A) { return stage_launch(ctx, PREC_F64, A); }

void set_stage(StageArgs& A, int stage, double dt) {
    A.stage = stage;
    A.dt = dt;
    A.cdt = stage == 2 ? 0.25 * dt : (stage == 3 ? (2.0 / 3.0) * dt : dt);
}

// Three fused stages of one SSP-RK3 step on the caller's U (Un = U on entry).
// Stage outputs ping-pong through workspace A and B; stage 3 writes U.
bsn_status f64_rk3(bsn_ctx* ctx, StageArgs base, double* U, double dt, const double* phi_per_stage[3],
                   unsigned long long* cfl_max, unsigned int* cfl_nan) {
    Geom G(base.nx, base.ny, base.nz);
    size_t bytes = sizeof(double) * (size_t)G.nelem();
    bsn_status st;
    double* A = (double*)slot(ctx, SLOT_A, bytes, &st); BSN_TRY(st);
    double* B = (double*)slot(ctx, SLOT_B, bytes, &st); BSN_TRY(st);
    double* in[3] = {U, A, B};
    double* out[3] = {A, B, U};
    for (int s = 0; s < 3; ++s) {
        StageArgs a = base;
        a.Uin = in[s]; a.Un = U; a.Uout = out[s]; a.mode = 0;
        set_stage(a, s + 1, dt);
        if (phi_per_stage) { a.phi = phi_per_stage[s]; a.use_sg = phi_per_stage[s] != nullptr; }
        a.cfl_max = (s == 2) ? cfl_max : nullptr;
        a.cfl_nan = cfl_nan;
        BSN_TRY(f64_launch_stage(ctx, a));
    }
    return f64_ghost_combine(ctx, U, B, nullptr, base.nx, base.ny, base.nz, base.bc, dt, nullptr, nullptr);
}

bsn_status f64_cfl_dt(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                      double gamma, double cfl, double* dt_out) {
    bsn_status st;
    unsigned long long* red = (unsigned long long*)slot(ctx, SLOT_RED, 64, &st); BSN_TRY(st);
    BSN_CUDA(ctx, cudaMemsetAsync(red, 0, 16, ctx->stream));
    long long n = (long long)nx * ny * nz;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
    prof_begin(ctx);
    cfl_kernel<<<blocks, 256, 0, ctx->stream>>>(U, nx, ny, nz, gamma, gamma - 1.0, 1.0 / dx, 1.0 / dy, 1.0 / dz,
                                                red, (unsigned int*)(red + 1));
    BSN_TRY(launch_check(ctx, "cfl_kernel"));
    return cfl_from_device(ctx, red, cfl, dt_out);
}

bsn_status f64_cfl_fold(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                        double gamma, unsigned long long* smax, unsigned int* nanflag) {
    long long n = (long long)nx * ny * nz;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
    prof_begin(ctx);
    cfl_kernel<<<blocks, 256, 0, ctx->stream>>>(U, nx, ny, nz, gamma, gamma - 1.0, 1.0 / dx, 1.0 / dy, 1.0 / dz, smax,
                                                nanflag);
    return launch_check(ctx, "cfl_kernel");
}

bsn_status cfl_from_device(bsn_ctx* ctx, const unsigned long long* red, double cfl, double* dt_out) {
    bsn_status st;
    unsigned long long* h = (unsigned long long*)pinned(ctx, 64, &st); BSN_TRY(st);
    BSN_CUDA(ctx, cudaMemcpyAsync(h, red, 16, cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    double smax;
    unsigned long long bits = h[0];
    memcpy(&smax, &bits, 8);
    unsigned int nanf = (unsigned int)(h[1] & 0xffffffffu);
    // reference: maximum() propagates NaN and `NaN > 0.0` is false -> Inf
    if (nanf) *dt_out = INFINITY;
    else *dt_out = smax > 0.0 ? cfl / smax : INFINITY;
    return BSN_OK;
}

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_fill_ghost_3d_f64(bsn_ctx* ctx, double* U, int nx, int ny, int nz, int bc) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U) return set_err(ctx, BSN_ERR_ARG, "U is null");
    if (bc == BSN_BC_PERIODIC && (nx < BSN_NG || ny < BSN_NG || nz < BSN_NG))
        return set_err(ctx, BSN_ERR_ARG, "periodic ghost fill needs n >= 3 per axis");
    return f64_fill_ghosts(ctx, U, nx, ny, nz, bc);
}

extern "C" bsn_status bsn_apply_floors_3d_f64(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double rho_floor,
                                              double P_floor, double gamma) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U) return set_err(ctx, BSN_ERR_ARG, "U is null");
    return f64_floors(ctx, U, nx, ny, nz, rho_floor, P_floor, gamma);
}

extern "C" bsn_status bsn_euler3d_rhs_f64(bsn_ctx* ctx, double* dU, double* Fx, double* Fy, double* Fz, double* U,
                                          int nx, int ny, int nz, double dx, double dy, double dz, double gamma,
                                          int bc, double rho_floor, double P_floor, int fill_ghosts) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || !dU) return set_err(ctx, BSN_ERR_ARG, "U and dU must be non-null");
    if (bc != BSN_BC_OUTFLOW && bc != BSN_BC_PERIODIC) return set_err(ctx, BSN_ERR_ARG, "bad bc %d", bc);
    Geom G(nx, ny, nz);
    if (fill_ghosts) BSN_TRY(f64_fill_ghosts(ctx, U, nx, ny, nz, bc));
    long long X = nx + 6, Y = ny + 6, Z = nz + 6;
    if (Fx) BSN_CUDA(ctx, cudaMemsetAsync(Fx, 0, sizeof(double) * 5 * (X + 1) * Y * Z, ctx->stream));
    if (Fy) BSN_CUDA(ctx, cudaMemsetAsync(Fy, 0, sizeof(double) * 5 * X * (Y + 1) * Z, ctx->stream));
    if (Fz) BSN_CUDA(ctx, cudaMemsetAsync(Fz, 0, sizeof(double) * 5 * X * Y * (Z + 1), ctx->stream));
    BSN_CUDA(ctx, cudaMemsetAsync(dU, 0, sizeof(double) * G.nelem(), ctx->stream));
    StageArgs A;
    stage_args_init(A, nx, ny, nz, dx, dy, dz, gamma, bc, rho_floor, P_floor);
    A.Uin = U;
    A.Gh = U;   // ghosts are whatever U holds (filled above or by the caller)
    A.dU = dU;
    A.F[0] = Fx; A.F[1] = Fy; A.F[2] = Fz;
    A.mode = 1;
    BSN_TRY(f64_launch_stage(ctx, A));
    // euler3d_rhs! floors U in place; the stage kernel floored its staged copies
    return f64_floors(ctx, U, nx, ny, nz, rho_floor, P_floor, gamma);
}

extern "C" bsn_status bsn_euler3d_step_f64(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double dx, double dy,
                                           double dz, double dt, double gamma, int bc, double rho_floor,
                                           double P_floor) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U) return set_err(ctx, BSN_ERR_ARG, "U is null");
    if (bc != BSN_BC_OUTFLOW && bc != BSN_BC_PERIODIC) return set_err(ctx, BSN_ERR_ARG, "bad bc %d", bc);
    if (bc == BSN_BC_PERIODIC && (nx < BSN_NG || ny < BSN_NG || nz < BSN_NG))
        return set_err(ctx, BSN_ERR_ARG, "periodic boundaries need n >= 3 per axis");
    StageArgs A;
    stage_args_init(A, nx, ny, nz, dx, dy, dz, gamma, bc, rho_floor, P_floor);
    return f64_rk3(ctx, A, U, dt, nullptr, nullptr, nullptr);
}

extern "C" bsn_status bsn_cfl_dt_3d_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy,
                                        double dz, double gamma, double cfl, double* dt_out) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || !dt_out) return set_err(ctx, BSN_ERR_ARG, "U and dt_out must be non-null");
    return f64_cfl_dt(ctx, U, nx, ny, nz, dx, dy, dz, gamma, cfl, dt_out);
}
