// tma_host.cu -- host side of the TMA staging (tma.cuh): tensor-map encoding
// of a stage input, the per-device error word of the bounded copy waits, and
// the switch between TMA staging and the plain loader.
#include <mutex>

#include "hydro_f64.cuh"
#include "tma.cuh"

namespace bsn {
namespace tma {

// set by a copy wait that ran out (bit 0); one word per device, read and
// cleared by check_error
static __device__ unsigned int g_tma_err;

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeFn encode_fn() {
    static std::once_flag once;
    static EncodeFn fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// The context's error word (looked up with the context's device current, at
// context creation; null leaves TMA staging off for the context).
void init_ctx(bsn_ctx* ctx) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tma_err) != cudaSuccess || !encode_fn()) {
        cudaGetLastError();
        ctx->tma_on = 0;
        ctx->tma_err = nullptr;
        return;
    }
    ctx->tma_err = (unsigned int*)p;
}

static bool encode(CUtensorMap* map, const double* base, const cuuint64_t dims[3], const cuuint64_t strides[2],
                   cuuint32_t bx, cuuint32_t by, cuuint32_t bz) {
    const cuuint32_t box[3] = {bx, by, bz};
    const cuuint32_t estr[3] = {1, 1, 1};
    return encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims, strides, box, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool build_maps(bsn_ctx* ctx, const f64::StageArgs& A, int TX, int TY, int TZ, int AY, int AZ, int YZ, int ZY,
                Maps& M) {
    if (!ctx->tma_on || !ctx->tma_now || !ctx->tma_err || A.Gh || !A.Uin) return false;
    if (A.nx % TX || A.ny % TY || A.nz % TZ || (A.nx & 1) || ((uintptr_t)A.Uin & 15)) return false;
    const cuuint64_t NXT = A.nx + 2 * BSN_NG, NYT = A.ny + 2 * BSN_NG, NZT = A.nz + 2 * BSN_NG;
    const cuuint64_t dims[3] = {5 * NXT, NYT, NZT};
    const cuuint64_t strides[2] = {5 * NXT * 8, 5 * NXT * NYT * 8};   // multiples of 16 since nx is even
    if (!encode(&M.a, A.Uin, dims, strides, 5 * (TX + 6), AY, AZ)) return false;
    if (!encode(&M.y, A.Uin, dims, strides, 5 * (TX + 2), 3, YZ)) return false;
    if (!encode(&M.z, A.Uin, dims, strides, 5 * (TX + 2), ZY, 3)) return false;
    M.err = ctx->tma_err;
    return true;
}

// BSN_ERR_TIMEOUT (and the word cleared) when a copy wait ran out since the
// last check; synchronises the context's stream.
bsn_status check_error(bsn_ctx* ctx) {
    if (!ctx->tma_err) return BSN_OK;
    unsigned int v = 0;
    BSN_CUDA(ctx, cudaMemcpyAsync(&v, ctx->tma_err, sizeof(v), cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (!v) return BSN_OK;
    BSN_CUDA(ctx, cudaMemsetAsync(ctx->tma_err, 0, sizeof(v), ctx->stream));
    return set_err(ctx, BSN_ERR_TIMEOUT, "a TMA copy of the stage kernel did not arrive within its wait bound");
}

}  // namespace tma

void run_state_free(bsn_ctx* ctx);             // run_steps.cu
void fmr_run_state_free(bsn_ctx* ctx);         // fmr_f64.cu
void fmrN_state_free(bsn_ctx* ctx);            // fmr_nlevel.cu
void coupled_run_state_free(bsn_ctx* ctx);     // coupled_run.cu
void coupled_nested_state_free(bsn_ctx* ctx);  // coupled_run.cu
void relax_state_free(bsn_ctx* ctx);           // relax.cu

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_ctx_set_tma(bsn_ctx* ctx, int on) {
    if (!ctx) return BSN_ERR_ARG;
    if (on && !ctx->tma_err) return set_err(ctx, BSN_ERR_UNSUPPORTED, "TMA staging is unavailable on this device");
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->tma_on = on ? 1 : 0;
    // captured step graphs hold the kernels chosen before the switch
    run_state_free(ctx);
    fmr_run_state_free(ctx);
    fmrN_state_free(ctx);
    coupled_run_state_free(ctx);
    coupled_nested_state_free(ctx);
    relax_state_free(ctx);
    ctx->tile_choice.clear();
    ctx->tile_last.clear();
    ctx->settled.clear();
    return BSN_OK;
}

extern "C" int bsn_ctx_get_tma(const bsn_ctx* ctx) { return ctx ? ctx->tma_on : 0; }
