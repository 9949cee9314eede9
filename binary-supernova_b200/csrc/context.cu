// context.cu -- bsn_ctx lifetime, error reporting and the reusable workspace.
#include <cstdarg>
#include <cstring>

#include "bsn_internal.cuh"

namespace bsn {

bsn_status set_err(bsn_ctx* ctx, bsn_status code, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return code;
}

bsn_status cuda_check(bsn_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return BSN_OK;
    return set_err(ctx, BSN_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

void prof_begin(bsn_ctx* ctx) {
    if (!ctx->profiling) return;
    cudaEvent_t a;
    if (cudaEventCreate(&a) != cudaSuccess) return;
    cudaEventRecord(a, ctx->stream);
    ctx->pending_start = a;
}

bsn_status launch_check(bsn_ctx* ctx, const char* what) {
    ctx->launches += 1;
    if (ctx->profiling && ctx->pending_start) {
        cudaEvent_t b;
        if (cudaEventCreate(&b) == cudaSuccess) {
            cudaEventRecord(b, ctx->stream);
            ctx->recs.push_back({what, ctx->pending_start, b});
        }
        ctx->pending_start = nullptr;
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return BSN_OK;
    return set_err(ctx, BSN_ERR_CUDA, "launch %s: %s", what, cudaGetErrorString(e));
}

void* slot(bsn_ctx* ctx, int s, size_t bytes, bsn_status* st) {
    *st = BSN_OK;
    if ((int)ctx->slot_ptr.size() <= s) {
        ctx->slot_ptr.resize(s + 1, nullptr);
        ctx->slot_bytes.resize(s + 1, 0);
    }
    if (bytes == 0) bytes = 256;
    if (ctx->slot_bytes[s] >= bytes) return ctx->slot_ptr[s];
    if (ctx->slot_ptr[s]) {
        // the stream may still use the old buffer
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->slot_ptr[s]);
        ctx->slot_ptr[s] = nullptr;
        ctx->slot_bytes[s] = 0;
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *st = set_err(ctx, BSN_ERR_NOMEM, "workspace slot %d: cudaMalloc(%zu) failed: %s", s, bytes,
                      cudaGetErrorString(e));
        return nullptr;
    }
    ctx->slot_ptr[s] = p;
    ctx->slot_bytes[s] = bytes;
    return p;
}

void* pinned(bsn_ctx* ctx, size_t bytes, bsn_status* st) {
    *st = BSN_OK;
    if (ctx->pinned_bytes >= bytes) return ctx->pinned;
    if (ctx->pinned) {
        cudaStreamSynchronize(ctx->stream);
        cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
    }
    cudaError_t e = cudaMallocHost(&ctx->pinned, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *st = set_err(ctx, BSN_ERR_NOMEM, "pinned host buffer (%zu B): %s", bytes, cudaGetErrorString(e));
        return nullptr;
    }
    ctx->pinned_bytes = bytes;
    return ctx->pinned;
}

void fft_state_free(bsn_ctx* ctx);   // poisson.cu
void fft32_state_free(bsn_ctx* ctx);   // poisson_f32.cu
void run_state_free(bsn_ctx* ctx);   // run_steps.cu
void learned_state_free(bsn_ctx* ctx);   // learned.cu
void fmr_run_state_free(bsn_ctx* ctx);   // fmr_f64.cu
void fmrN_state_free(bsn_ctx* ctx);      // fmr_nlevel.cu
void coupled_run_state_free(bsn_ctx* ctx);   // coupled_run.cu
void coupled_nested_state_free(bsn_ctx* ctx);   // coupled_run.cu
void relax_state_free(bsn_ctx* ctx);     // relax.cu
void ckpt_state_free(bsn_ctx* ctx);      // h5io.cu

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_ctx_create(bsn_ctx** out, int device, void* stream) {
    if (!out) return BSN_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return BSN_ERR_CUDA;
    }
    if (device < 0 || device >= n) return BSN_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return BSN_ERR_CUDA;
    bsn_ctx* c = new bsn_ctx();
    c->device = device;
    c->stream = (cudaStream_t)stream;
    c->slot_ptr.assign(SLOT_COUNT, nullptr);
    c->slot_bytes.assign(SLOT_COUNT, 0);
    tma::init_ctx(c);
    *out = c;
    return BSN_OK;
}

extern "C" bsn_status bsn_ctx_destroy(bsn_ctx* ctx) {
    if (!ctx) return BSN_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (void* p : ctx->slot_ptr)
        if (p) cudaFree(p);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    fft_state_free(ctx);
    fft32_state_free(ctx);
    run_state_free(ctx);
    learned_state_free(ctx);
    fmr_run_state_free(ctx);
    fmrN_state_free(ctx);
    coupled_run_state_free(ctx);
    coupled_nested_state_free(ctx);
    relax_state_free(ctx);
    ckpt_state_free(ctx);
    for (auto& r : ctx->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    delete ctx;
    return BSN_OK;
}

extern "C" bsn_status bsn_ctx_set_stream(bsn_ctx* ctx, void* stream) {
    if (!ctx) return BSN_ERR_ARG;
    ctx->stream = (cudaStream_t)stream;
    return BSN_OK;
}

extern "C" bsn_status bsn_ctx_set_stiff_guard(bsn_ctx* ctx, int on) {
    if (!ctx) return BSN_ERR_ARG;
    BSN_TRY(cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"));
    ctx->stiff_guard = on ? 1 : 0;
    // the captured time-loop graphs hold the kernels chosen before
    bsn::run_state_free(ctx);
    bsn::fmr_run_state_free(ctx);
    bsn::fmrN_state_free(ctx);
    bsn::relax_state_free(ctx);
    return BSN_OK;
}

extern "C" bsn_status bsn_ctx_synchronize(bsn_ctx* ctx) {
    if (!ctx) return BSN_ERR_ARG;
    BSN_TRY(cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"));
    return tma::check_error(ctx);
}

extern "C" const char* bsn_last_error(const bsn_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" const char* bsn_version(void) { return "libbsn 0.1 (sm_100a)"; }

extern "C" long long bsn_ctx_launch_count(const bsn_ctx* ctx) { return ctx ? ctx->launches : -1; }

extern "C" bsn_status bsn_ctx_set_profiling(bsn_ctx* ctx, int on) {
    if (!ctx) return BSN_ERR_ARG;
    cudaStreamSynchronize(ctx->stream);
    for (auto& r : ctx->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    ctx->recs.clear();
    ctx->profiling = on != 0;
    return BSN_OK;
}

extern "C" bsn_status bsn_ctx_kernel_stats(bsn_ctx* ctx, const char* name, double* total_ms, long long* count) {
    if (!ctx || !name || !total_ms || !count) return BSN_ERR_ARG;
    BSN_TRY(cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"));
    double t = 0.0;
    long long n = 0;
    for (auto& r : ctx->recs) {
        if (r.name != name) continue;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) { t += ms; ++n; }
    }
    *total_ms = t;
    *count = n;
    return BSN_OK;
}
