// poisson.cu -- isolated-boundary Poisson solve with hand-written batched FFTs
// (Hockney-Eastwood zero padding; src/self_gravity.jl:35-76).
//
//   Phi = dV * Re( IFFT( FFT(K) . FFT(rho_pad) ) )[0:n, 0:n, 0:n]
//
// on the doubled grid N = 2n per axis, K = -1/sqrt(r^2 + eps^2) with folded
// indices.  B200 pipeline (power-of-two N per axis):
//   * K is even along every axis, so Khat is real and even: it is built once
//     per grid on the device ((nx+1)(ny+1)(nz+1) reals, dV/(N1 N2 N3) folded
//     in) and cached in the context -- the reference rebuilds K on the host
//     and uploads it on every call;
//   * forward passes skip the zero padding: x transforms only the n^2 rows
//     that hold density and keeps the n+1 non-redundant frequencies of the
//     real input, y transforms only the n z-planes that hold data;
//   * one kernel does the z forward transform, the multiplication by Khat and
//     the z inverse transform per line (decimation in frequency then in time,
//     so no bit reversal is needed between them) and keeps only the n output
//     planes the solution needs; the full padded spectrum never reaches HBM;
//   * inverse y and x passes produce only the first octant.
// The solve's transforms are register-resident self-sorting FFTs over
// batches of lines (fft_lines.cuh) whose neighbouring elements are contiguous
// in HBM, so loads and stores are coalesced for all three axes; Khat's
// one-off transforms are radix-2 FFTs in shared memory.
#include <cmath>
#include <map>

#include "fft_lines.cuh"
#include "poisson.cuh"

namespace bsn {
namespace fft {

constexpr int NT = 256;
constexpr int SMEM_COMPLEX = 4096;   // complex doubles of line storage per CTA (64 KiB)

struct Twiddles {
    double2* d = nullptr;   // exp(-2 pi i t / N), t < N/2
};

struct State {
    std::map<int, Twiddles> tw;
    double* khat = nullptr;
    size_t khat_bytes = 0;
    int knx = 0, kny = 0, knz = 0;
    double kdx = 0, kdy = 0, kdz = 0;
};

// ---- Khat: three passes over K restricted to the non-negative octant ------
// pass a: lines along x for (my <= ny, mz <= nz), K generated on the fly
__global__ void khat_x_kernel(double* T1, int nx, int ny, int nz, double dx, double dy, double dz, double eps2,
                              int logn, int lines, const double2* tw) {
    extern __shared__ double2 sm[];
    const int N = 1 << logn;
    double2* stw = sm;
    double2* s = sm + (N >> 1);
    load_twiddles(stw, tw, logn);
    long long nrows = (long long)(ny + 1) * (nz + 1);
    long long row0 = (long long)blockIdx.x * lines;
    for (int t = threadIdx.x; t < lines * N; t += blockDim.x) {
        int l = t / N, m = t - l * N;
        long long row = row0 + l;
        double v = 0.0;
        if (row < nrows) {
            int my = (int)(row % (ny + 1)), mz = (int)(row / (ny + 1));
            double fi = (double)(m < nx ? m : m - N);
            double fj = (double)(my < ny ? my : my - 2 * ny);
            double fk = (double)(mz < nz ? mz : mz - 2 * nz);
            double r2 = (fi * dx) * (fi * dx) + (fj * dy) * (fj * dy) + (fk * dz) * (fk * dz);
            v = -1.0 / sqrt(r2 + eps2);
        }
        s[l * N + bitrev(m, logn)] = make_double2(v, 0.0);
    }
    fft_dit(s, stw, lines, logn, false);
    for (int t = threadIdx.x; t < lines * (nx + 1); t += blockDim.x) {
        int l = t / (nx + 1), kx = t - l * (nx + 1);
        long long row = row0 + l;
        if (row < nrows) T1[kx + (long long)(nx + 1) * row] = s[l * N + kx].x;
    }
}

// passes b, c: even real lines along an axis of stride `estride` with `nhalf`
// stored samples (0..n); output the real part of frequencies 0..n, times `scale`.
__global__ void khat_even_kernel(const double* in, double* out, int nkx, long long nouter, long long estride,
                                 long long ostride, int n, double scale, int logn, int lines, const double2* tw) {
    extern __shared__ double2 sm[];
    const int N = 1 << logn;
    double2* stw = sm;
    double2* s = sm + (N >> 1);
    load_twiddles(stw, tw, logn);
    int nbx = (nkx + lines - 1) / lines;
    long long outer = blockIdx.x / nbx;
    int kx0 = (int)(blockIdx.x % nbx) * lines;
    for (int t = threadIdx.x; t < lines * N; t += blockDim.x) {
        int l = t % lines, m = t / lines;
        int kx = kx0 + l;
        double v = 0.0;
        if (kx < nkx && outer < nouter) {
            int mf = m <= n ? m : N - m;
            v = in[kx + outer * ostride + mf * estride];
        }
        s[l * N + bitrev(m, logn)] = make_double2(v, 0.0);
    }
    fft_dit(s, stw, lines, logn, false);
    for (int t = threadIdx.x; t < lines * (n + 1); t += blockDim.x) {
        int l = t % lines, k = t / lines;
        int kx = kx0 + l;
        if (kx < nkx && outer < nouter) out[kx + outer * ostride + k * estride] = s[l * N + k].x * scale;
    }
}

int ilog2(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}
bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

State* state(bsn_ctx* ctx) {
    if (!ctx->fft_state) ctx->fft_state = new State();
    return (State*)ctx->fft_state;
}

bsn_status twiddles(bsn_ctx* ctx, int N, const double2** out) {
    State* S = state(ctx);
    auto it = S->tw.find(N);
    if (it != S->tw.end()) { *out = it->second.d; return BSN_OK; }
    std::vector<double2> h(N / 2 > 0 ? N / 2 : 1);
    for (int t = 0; t < N / 2; ++t) {
        long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)N;
        h[t] = make_double2((double)cosl(a), (double)sinl(a));
    }
    double2* d = nullptr;
    BSN_CUDA(ctx, cudaMalloc(&d, sizeof(double2) * h.size()));
    BSN_CUDA(ctx, cudaMemcpy(d, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice));
    S->tw[N] = Twiddles{d};
    *out = d;
    return BSN_OK;
}

int lines_for(int N) { return std::max(1, std::min(64, SMEM_COMPLEX / N)); }
size_t smem_for(int N, int lines) { return sizeof(double2) * ((size_t)lines * N + N / 2); }

bsn_status set_smem(bsn_ctx* ctx) {
    static bool done[64] = {false};
    int dev = ctx->device & 63;
    if (done[dev]) return BSN_OK;
    int bytes = (int)(sizeof(double2) * (SMEM_COMPLEX + 2048));
    const void* ks[] = {(const void*)khat_x_kernel, (const void*)khat_even_kernel};
    for (const void* k : ks)
        BSN_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    done[dev] = true;
    return BSN_OK;
}

// Khat for the grid, cached: real (nx+1)(ny+1)(nz+1) with dV/(N1 N2 N3) folded
// in (the allocation holds a second octant used as scratch while building).
bsn_status khat(bsn_ctx* ctx, int nx, int ny, int nz, double dx, double dy, double dz, const double** out) {
    State* S = state(ctx);
    if (S->khat && S->knx == nx && S->kny == ny && S->knz == nz && S->kdx == dx && S->kdy == dy && S->kdz == dz) {
        *out = S->khat;
        return BSN_OK;
    }
    int N1 = 2 * nx, N2 = 2 * ny, N3 = 2 * nz;
    size_t nk = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    size_t bytes = sizeof(double) * (2 * nk);
    if (S->khat && S->khat_bytes < bytes) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(S->khat);
        S->khat = nullptr;
    }
    if (!S->khat) {
        BSN_CUDA(ctx, cudaMalloc(&S->khat, bytes));
        S->khat_bytes = bytes;
    }
    double* K = S->khat;
    double* T = K + nk;   // temporary octant buffer
    const double2 *t1, *t2, *t3;
    BSN_TRY(twiddles(ctx, N1, &t1));
    BSN_TRY(twiddles(ctx, N2, &t2));
    BSN_TRY(twiddles(ctx, N3, &t3));
    double eps2 = std::pow(dx * dy * dz, 2.0 / 3.0);
    double scale = (dx * dy * dz) / ((double)N1 * (double)N2 * (double)N3);
    int l1 = lines_for(N1), l2 = lines_for(N2), l3 = lines_for(N3);
    long long rows = (long long)(ny + 1) * (nz + 1);
    prof_begin(ctx);
    khat_x_kernel<<<grid1d(rows, l1), NT, smem_for(N1, l1), ctx->stream>>>(T, nx, ny, nz, dx, dy, dz, eps2,
                                                                           ilog2(N1), l1, t1);
    BSN_TRY(launch_check(ctx, "khat_x_kernel"));
    // y: lines along y (stride nx+1) for each (kx, mz); T -> K
    {
        int nbx = (nx + 1 + l2 - 1) / l2;
        prof_begin(ctx);
        khat_even_kernel<<<(unsigned)(nbx * (nz + 1)), NT, smem_for(N2, l2), ctx->stream>>>(
            T, K, nx + 1, nz + 1, nx + 1, (long long)(nx + 1) * (ny + 1), ny, 1.0, ilog2(N2), l2, t2);
        BSN_TRY(launch_check(ctx, "khat_even_kernel"));
    }
    // z: lines along z (stride (nx+1)(ny+1)) for each (kx, ky); K -> T (scaled)
    {
        int nbx = (nx + 1 + l3 - 1) / l3;
        prof_begin(ctx);
        khat_even_kernel<<<(unsigned)(nbx * (ny + 1)), NT, smem_for(N3, l3), ctx->stream>>>(
            K, T, nx + 1, ny + 1, (long long)(nx + 1) * (ny + 1), nx + 1, nz, scale, ilog2(N3), l3, t3);
        BSN_TRY(launch_check(ctx, "khat_even_kernel"));
    }
    BSN_CUDA(ctx, cudaMemcpyAsync(K, T, sizeof(double) * nk, cudaMemcpyDeviceToDevice, ctx->stream));
    S->knx = nx; S->kny = ny; S->knz = nz; S->kdx = dx; S->kdy = dy; S->kdz = dz;
    *out = K;
    return BSN_OK;
}

bsn_status solve(bsn_ctx* ctx, RhoSrc src, double dx, double dy, double dz, double* phi) {
    int nx = src.nx, ny = src.ny, nz = src.nz;
    if (!pow2(nx) || !pow2(ny) || !pow2(nz) || nx < 2 || ny < 2 || nz < 2)
        return set_err(ctx, BSN_ERR_UNSUPPORTED, "FFT Poisson solve needs power-of-two sizes >= 2 (got %d,%d,%d)",
                       nx, ny, nz);
    if (2 * std::max(nx, std::max(ny, nz)) > SMEM_COMPLEX)
        return set_err(ctx, BSN_ERR_UNSUPPORTED, "FFT length above %d", SMEM_COMPLEX);
    BSN_TRY(set_smem(ctx));
    int N1 = 2 * nx, N2 = 2 * ny, N3 = 2 * nz;
    const double* K;
    BSN_TRY(khat(ctx, nx, ny, nz, dx, dy, dz, &K));
    const double2 *t1, *t2, *t3;
    BSN_TRY(twiddles(ctx, N1, &t1));
    BSN_TRY(twiddles(ctx, N2, &t2));
    BSN_TRY(twiddles(ctx, N3, &t3));
    size_t w1 = (size_t)(nx + 1) * ny * nz, w2 = (size_t)(nx + 1) * N2 * nz;
    bsn_status st;
    double2* W1 = (double2*)slot(ctx, SLOT_FFT0, sizeof(double2) * w1, &st); BSN_TRY(st);
    double2* W2 = (double2*)slot(ctx, SLOT_FFT1, sizeof(double2) * w2, &st); BSN_TRY(st);
    return solve_lines<double2>(ctx, src, K, t1, t2, t3, W1, W2, phi);
}

}  // namespace fft

void fft_state_free(bsn_ctx* ctx) {
    if (!ctx->fft_state) return;
    fft::State* S = (fft::State*)ctx->fft_state;
    for (auto& kv : S->tw) cudaFree(kv.second.d);
    if (S->khat) cudaFree(S->khat);
    delete S;
    ctx->fft_state = nullptr;
}

bsn_status poisson_khat64(bsn_ctx* ctx, int nx, int ny, int nz, double dx, double dy, double dz, const double** K) {
    BSN_TRY(fft::set_smem(ctx));
    return fft::khat(ctx, nx, ny, nz, dx, dy, dz, K);
}

bsn_status poisson_prepare(bsn_ctx* ctx, int nx, int ny, int nz, double dx, double dy, double dz) {
    if (!fft::pow2(nx) || !fft::pow2(ny) || !fft::pow2(nz) || nx < 2 || ny < 2 || nz < 2)
        return set_err(ctx, BSN_ERR_UNSUPPORTED, "FFT Poisson solve needs power-of-two sizes >= 2 (got %d,%d,%d)",
                       nx, ny, nz);
    BSN_TRY(fft::set_smem(ctx));
    const double* K;
    BSN_TRY(fft::khat(ctx, nx, ny, nz, dx, dy, dz, &K));
    const double2* t;
    BSN_TRY(fft::twiddles(ctx, 2 * nx, &t));
    BSN_TRY(fft::twiddles(ctx, 2 * ny, &t));
    BSN_TRY(fft::twiddles(ctx, 2 * nz, &t));
    bsn_status st;
    slot(ctx, SLOT_FFT0, sizeof(double2) * (size_t)(nx + 1) * ny * nz, &st); BSN_TRY(st);
    slot(ctx, SLOT_FFT1, sizeof(double2) * (size_t)(nx + 1) * (2 * ny) * nz, &st); BSN_TRY(st);
    return BSN_OK;
}

bsn_status poisson_solve(bsn_ctx* ctx, const double* rho, int nx, int ny, int nz, double dx, double dy, double dz,
                         double* phi) {
    if (!rho || !phi) return set_err(ctx, BSN_ERR_ARG, "rho and phi must be non-null");
    fft::RhoSrc s{rho, nullptr, nx, ny, nz, -1.0};
    return fft::solve(ctx, s, dx, dy, dz, phi);
}

bsn_status poisson_from_state(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                              double rho_floor, double* phi) {
    fft::RhoSrc s{nullptr, U, nx, ny, nz, rho_floor};
    return fft::solve(ctx, s, dx, dy, dz, phi);
}

// coupled_step! with self-gravity: each stage solves Poisson on the floored
// density of its input (add_self_gravity_source! after euler3d_rhs!).
bsn_status f64_rk3_selfgrav(bsn_ctx* ctx, f64::StageArgs base, double* U, double dt) {
    Geom G(base.nx, base.ny, base.nz);
    size_t bytes = sizeof(double) * (size_t)G.nelem();
    bsn_status st;
    double* A = (double*)slot(ctx, SLOT_A, bytes, &st); BSN_TRY(st);
    double* B = (double*)slot(ctx, SLOT_B, bytes, &st); BSN_TRY(st);
    double* phi = (double*)slot(ctx, SLOT_PHI, sizeof(double) * (size_t)base.nx * base.ny * base.nz, &st);
    BSN_TRY(st);
    double* in[3] = {U, A, B};
    double* out[3] = {A, B, U};
    for (int s = 0; s < 3; ++s) {
        BSN_TRY(poisson_from_state(ctx, in[s], base.nx, base.ny, base.nz, base.dx, base.dy, base.dz, base.rho_floor,
                                   phi));
        f64::StageArgs a = base;
        a.Uin = in[s]; a.Un = U; a.Uout = out[s]; a.mode = 0;
        set_stage(a, s + 1, dt);
        a.phi = phi; a.use_sg = 1;
        BSN_TRY(f64_launch_stage(ctx, a));
    }
    return f64_ghost_combine(ctx, U, B, nullptr, base.nx, base.ny, base.nz, base.bc, dt);
}

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_solve_poisson_isolated_f64(bsn_ctx* ctx, const double* rho, int nx, int ny, int nz, double dx,
                                                     double dy, double dz, double* phi) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    return poisson_solve(ctx, rho, nx, ny, nz, dx, dy, dz, phi);
}

// ---- z-slab decomposition of solve_poisson_isolated -------------------------
// A rank holding planes [z0, z0 + nzl) of the density runs slab_forward on
// them, sends W2's ky range of every rank to that rank (an all-to-all), runs
// slab_zconv on the z lines of its own ky range (all nz planes, in z order),
// sends each rank's z range back and runs slab_inverse on its planes.  W2 and
// T are interleaved complex doubles: W2[kx + (nx+1)*(ky + 2ny*z)], z < nzl;
// T[kx + (nx+1)*(kyl + nky*z)], z < nz.

static bsn_status slab_check(bsn_ctx* ctx, int nx, int ny, int nz) {
    if (!ctx) return BSN_ERR_ARG;
    if (!fft::pow2(nx) || !fft::pow2(ny) || nx < 2 || ny < 2 || nz < 1)
        return set_err(ctx, BSN_ERR_UNSUPPORTED, "slab FFT needs power-of-two nx, ny >= 2 and nz >= 1 (got %d,%d,%d)",
                       nx, ny, nz);
    if (2 * std::max(nx, ny) > fft::SMEM_COMPLEX) return set_err(ctx, BSN_ERR_UNSUPPORTED, "FFT length above %d",
                                                                 fft::SMEM_COMPLEX);
    return BSN_OK;
}

extern "C" bsn_status bsn_poisson_slab_forward_f64(bsn_ctx* ctx, const double* rho, int nx, int ny, int nzl,
                                                   double* W2) {
    BSN_TRY(slab_check(ctx, nx, ny, nzl));
    if (!rho || !W2) return set_err(ctx, BSN_ERR_ARG, "rho and W2 must be non-null");
    const double2 *t1, *t2;
    BSN_TRY(fft::twiddles(ctx, 2 * nx, &t1));
    BSN_TRY(fft::twiddles(ctx, 2 * ny, &t2));
    bsn_status st;
    double2* W1 = (double2*)slot(ctx, SLOT_FFT0, sizeof(double2) * (size_t)(nx + 1) * ny * nzl, &st); BSN_TRY(st);
    fft::RhoSrc src{rho, nullptr, nx, ny, nzl, -1.0};
    return fft::slab_forward_lines<double2>(ctx, src, t1, t2, W1, (double2*)W2);
}

extern "C" bsn_status bsn_poisson_slab_zconv_f64(bsn_ctx* ctx, double* T, int nx, int ny, int nz, int ky0, int nky,
                                                 double dx, double dy, double dz) {
    BSN_TRY(slab_check(ctx, nx, ny, nz));
    if (!fft::pow2(nz) || nz < 2 || 2 * nz > fft::SMEM_COMPLEX)
        return set_err(ctx, BSN_ERR_UNSUPPORTED, "global nz must be a power of two in [2, %d] (got %d)",
                       fft::SMEM_COMPLEX / 2, nz);
    if (ky0 < 0 || nky < 0 || ky0 + nky > 2 * ny)
        return set_err(ctx, BSN_ERR_ARG, "ky range [%d, %d) outside [0, %d)", ky0, ky0 + nky, 2 * ny);
    if (nky > 0 && !T) return set_err(ctx, BSN_ERR_ARG, "T must be non-null");
    BSN_TRY(fft::set_smem(ctx));
    const double* K;
    BSN_TRY(fft::khat(ctx, nx, ny, nz, dx, dy, dz, &K));
    const double2* t3;
    BSN_TRY(fft::twiddles(ctx, 2 * nz, &t3));
    return fft::slab_zconv_lines<double2>(ctx, (double2*)T, K, t3, nx, ny, nz, ky0, nky);
}

extern "C" bsn_status bsn_poisson_slab_inverse_f64(bsn_ctx* ctx, const double* W2, int nx, int ny, int nzl,
                                                   double* phi) {
    BSN_TRY(slab_check(ctx, nx, ny, nzl));
    if (!W2 || !phi) return set_err(ctx, BSN_ERR_ARG, "W2 and phi must be non-null");
    const double2 *t1, *t2;
    BSN_TRY(fft::twiddles(ctx, 2 * nx, &t1));
    BSN_TRY(fft::twiddles(ctx, 2 * ny, &t2));
    bsn_status st;
    double2* W1 = (double2*)slot(ctx, SLOT_FFT0, sizeof(double2) * (size_t)(nx + 1) * ny * nzl, &st); BSN_TRY(st);
    return fft::slab_inverse_lines<double2>(ctx, (const double2*)W2, t1, t2, W1, phi, nx, ny, nzl);
}
