// fp_peak.cu -- measured FP64 and FP32 multiply-add throughput of this GPU,
// the denominators of the stencil kernels' FP-pipe fraction.  Every thread
// runs eight independent FMA chains x <- x*a + b (a, b set at run time, so
// nothing folds; the chains converge to b/(1-a), no overflow or subnormals),
// on a grid of 4 CTAs of 256 threads per SM.  One FMA counts as two flops;
// the packed FP32 form (fma.rn.f32x2) does two FMAs per instruction.
#include "bsn_internal.cuh"

namespace bsn {
namespace peak {

constexpr int NT = 256;

template <typename T>
__global__ void __launch_bounds__(NT) fma_chains(T* out, int iters, T a, T b) {
    T x[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = T(threadIdx.x + c) * T(1e-3);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) x[c] = fma(x[c], a, b);
    }
    T s = x[0];
#pragma unroll
    for (int c = 1; c < 8; ++c) s += x[c];
    if (s == T(-1.0)) out[0] = s;   // never true; keeps the chains live
}

__global__ void __launch_bounds__(NT) fma_chains_f32x2(float* out, int iters, float a, float b) {
    unsigned long long x[8];
    unsigned long long av, bv;
    asm("mov.b64 %0, {%1, %1};" : "=l"(av) : "f"(a));
    asm("mov.b64 %0, {%1, %1};" : "=l"(bv) : "f"(b));
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        float lo = (float)(threadIdx.x + c) * 1e-3f, hi = lo + 0.5f;
        asm("mov.b64 %0, {%1, %2};" : "=l"(x[c]) : "f"(lo), "f"(hi));
    }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[c]) : "l"(av), "l"(bv));
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x[c]));
        s += lo + hi;
    }
    if (s == -1.0f) out[0] = s;
}

}  // namespace peak
}  // namespace bsn

using namespace bsn;

// precision: 0 FP64, 1 FP32 (scalar FFMA), 2 FP32 packed (f32x2).  Writes the
// best of three timed launches (CUDA events on the context's stream) in
// TFLOP/s.  Synchronises the stream.
extern "C" bsn_status bsn_fp_peak(bsn_ctx* ctx, int precision, double* tflops) {
    if (!ctx || !tflops || precision < 0 || precision > 2) return BSN_ERR_ARG;
    int sms = 0;
    BSN_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const int grid = 4 * sms;
    const int iters = precision == 0 ? 65536 : 131072;   // a few ms per launch
    bsn_status st;
    double* out = (double*)slot(ctx, SLOT_RED, 64, &st); BSN_TRY(st);
    auto launch = [&]() {
        if (precision == 0)
            peak::fma_chains<double><<<grid, peak::NT, 0, ctx->stream>>>(out, iters, 0.999999, 1e-6);
        else if (precision == 1)
            peak::fma_chains<float><<<grid, peak::NT, 0, ctx->stream>>>((float*)out, iters, 0.9999f, 1e-4f);
        else
            peak::fma_chains_f32x2<<<grid, peak::NT, 0, ctx->stream>>>((float*)out, iters, 0.9999f, 1e-4f);
    };
    cudaEvent_t e0, e1;
    BSN_CUDA(ctx, cudaEventCreate(&e0));
    BSN_CUDA(ctx, cudaEventCreate(&e1));
    launch();   // warm-up
    float best = 0.f;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e0, ctx->stream);
        launch();
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r == 0 || ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BSN_TRY(launch_check(ctx, "fma_chains"));
    const double fmas = (double)grid * peak::NT * 8.0 * iters * (precision == 2 ? 2.0 : 1.0);
    *tflops = 2.0 * fmas / (best * 1e-3) / 1e12;
    return BSN_OK;
}
