// poisson_f32.cu -- the isolated Poisson solve with FP32 transforms (the
// precision form of the FFTs): the same five passes as the FP64 solve
// (fft_lines.cuh) on float2 lines, the FP64 Green's-function transform
// converted once to FP32 and cached, density in and potential out in FP64.
// Built with the fast-path flags (FMA contraction).
#include <map>
#include <vector>

#include "fft_lines.cuh"
#include "poisson.cuh"

namespace bsn {
namespace fft32 {

constexpr int MAX_LEN = 4096;   // longest padded line of the transforms (fft_lines.cuh)

struct State {
    std::map<int, float2*> tw;
    float* khat = nullptr;
    size_t khat_cap = 0;
    int knx = 0, kny = 0, knz = 0;
    double kdx = 0, kdy = 0, kdz = 0;
};

State* state(bsn_ctx* ctx) {
    if (!ctx->fft32_state) ctx->fft32_state = new State();
    return (State*)ctx->fft32_state;
}

bsn_status twiddles(bsn_ctx* ctx, int N, const float2** out) {
    State* S = state(ctx);
    auto it = S->tw.find(N);
    if (it != S->tw.end()) { *out = it->second; return BSN_OK; }
    std::vector<float2> h(N / 2 > 0 ? N / 2 : 1);
    for (int t = 0; t < N / 2; ++t) {
        long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)N;
        h[t] = make_float2((float)cosl(a), (float)sinl(a));
    }
    float2* d = nullptr;
    BSN_CUDA(ctx, cudaMalloc(&d, sizeof(float2) * h.size()));
    BSN_CUDA(ctx, cudaMemcpy(d, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice));
    S->tw[N] = d;
    *out = d;
    return BSN_OK;
}

__global__ void to_float_kernel(const double* in, float* out, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        out[t] = (float)in[t];
}

bsn_status khat(bsn_ctx* ctx, int nx, int ny, int nz, double dx, double dy, double dz, const float** out) {
    State* S = state(ctx);
    if (S->khat && S->knx == nx && S->kny == ny && S->knz == nz && S->kdx == dx && S->kdy == dy && S->kdz == dz) {
        *out = S->khat;
        return BSN_OK;
    }
    const double* K64;
    BSN_TRY(poisson_khat64(ctx, nx, ny, nz, dx, dy, dz, &K64));
    long long nk = (long long)(nx + 1) * (ny + 1) * (nz + 1);
    if (S->khat && S->khat_cap < (size_t)nk) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(S->khat);
        S->khat = nullptr;
    }
    if (!S->khat) {
        BSN_CUDA(ctx, cudaMalloc(&S->khat, sizeof(float) * nk));
        S->khat_cap = (size_t)nk;
    }
    prof_begin(ctx);
    to_float_kernel<<<(int)std::min<long long>((nk + 255) / 256, 148LL * 8), 256, 0, ctx->stream>>>(K64, S->khat, nk);
    BSN_TRY(launch_check(ctx, "khat_to_float_kernel"));
    S->knx = nx; S->kny = ny; S->knz = nz; S->kdx = dx; S->kdy = dy; S->kdz = dz;
    *out = S->khat;
    return BSN_OK;
}

bsn_status prepare(bsn_ctx* ctx, int nx, int ny, int nz, double dx, double dy, double dz, const float** K,
                   const float2* tw[3], float2** W1, float2** W2) {
    if (nx < 2 || ny < 2 || nz < 2 || (nx & (nx - 1)) || (ny & (ny - 1)) || (nz & (nz - 1)))
        return set_err(ctx, BSN_ERR_UNSUPPORTED, "FFT Poisson solve needs power-of-two sizes >= 2 (got %d,%d,%d)",
                       nx, ny, nz);
    if (2 * std::max(nx, std::max(ny, nz)) > MAX_LEN)
        return set_err(ctx, BSN_ERR_UNSUPPORTED, "FFT length above %d", MAX_LEN);
    BSN_TRY(khat(ctx, nx, ny, nz, dx, dy, dz, K));
    BSN_TRY(twiddles(ctx, 2 * nx, &tw[0]));
    BSN_TRY(twiddles(ctx, 2 * ny, &tw[1]));
    BSN_TRY(twiddles(ctx, 2 * nz, &tw[2]));
    bsn_status st;
    *W1 = (float2*)slot(ctx, SLOT_FFT0, sizeof(float2) * (size_t)(nx + 1) * ny * nz, &st); BSN_TRY(st);
    *W2 = (float2*)slot(ctx, SLOT_FFT1, sizeof(float2) * (size_t)(nx + 1) * (2 * ny) * nz, &st); BSN_TRY(st);
    return BSN_OK;
}

bsn_status solve(bsn_ctx* ctx, const fft::RhoSrc& src, double dx, double dy, double dz, double* phi) {
    const float* K;
    const float2* tw[3];
    float2 *W1, *W2;
    BSN_TRY(prepare(ctx, src.nx, src.ny, src.nz, dx, dy, dz, &K, tw, &W1, &W2));
    return fft::solve_lines<float2>(ctx, src, K, tw[0], tw[1], tw[2], W1, W2, phi);
}

}  // namespace fft32

void fft32_state_free(bsn_ctx* ctx) {
    if (!ctx->fft32_state) return;
    fft32::State* S = (fft32::State*)ctx->fft32_state;
    for (auto& kv : S->tw) cudaFree(kv.second);
    if (S->khat) cudaFree(S->khat);
    delete S;
    ctx->fft32_state = nullptr;
}

bsn_status poisson_prepare_f32(bsn_ctx* ctx, int nx, int ny, int nz, double dx, double dy, double dz) {
    const float* K;
    const float2* tw[3];
    float2 *W1, *W2;
    return fft32::prepare(ctx, nx, ny, nz, dx, dy, dz, &K, tw, &W1, &W2);
}

bsn_status poisson_solve_f32(bsn_ctx* ctx, const double* rho, int nx, int ny, int nz, double dx, double dy, double dz,
                             double* phi) {
    if (!rho || !phi) return set_err(ctx, BSN_ERR_ARG, "rho and phi must be non-null");
    fft::RhoSrc s{rho, nullptr, nx, ny, nz, -1.0};
    return fft32::solve(ctx, s, dx, dy, dz, phi);
}

bsn_status poisson_from_state_f32(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy,
                                  double dz, double rho_floor, double* phi) {
    fft::RhoSrc s{nullptr, U, nx, ny, nz, rho_floor};
    return fft32::solve(ctx, s, dx, dy, dz, phi);
}

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_solve_poisson_isolated_f32(bsn_ctx* ctx, const double* rho, int nx, int ny, int nz,
                                                     double dx, double dy, double dz, double* phi) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    return poisson_solve_f32(ctx, rho, nx, ny, nz, dx, dy, dz, phi);
}
