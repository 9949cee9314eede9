// cfl_noalloc.cu -- cfl_dt_3d for callers that must not allocate GPU memory.
//
// bsn_cfl_dt_3d_f64 reduces through a workspace the context grows with
// cudaMalloc on first use.  Some callers cannot allow that: a host runtime
// that owns a fixed device-memory pool (for example a Julia process whose
// CUDA.jl pool has reserved the device, or a job that pre-sizes all of its
// memory at start-up and treats any later allocation failure as fatal) needs
// a dt reduction that never asks the driver for memory.  This variant keeps
// its scratch in a file-scope static device array instead:
//
//   * capacity: one partial maximum per 2048 active cells, 65536 partials,
//     so grids of at most 134,217,728 active cells (512^3) are accepted; larger
//     grids are rejected with BSN_ERR_UNSUPPORTED before anything is launched;
//   * the array occupies 512 KiB on every GPU that loads the library, until
//     the process exits.  The library is built without relocatable device
//     code, so this file is a module of its own, and under CUDA's lazy module
//     loading (the default since CUDA 12.2) the driver reserves the array on
//     a device only when this file's module is first used there: at the first
//     call of this entry point on that device.  A caller whose pool will
//     later reserve the whole device should make one warm-up call at start-up,
//     before the pool takes its memory, or run with CUDA_MODULE_LOADING=EAGER;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress, with that device current) and caches it per
//     device; this first call should come before any stream capture.  The
//     device is the context's: a call made while another device is current
//     is rejected with BSN_ERR_ARG, since the context's stream and the array
//     of the current device would then belong to different GPUs;
//   * every call shares the array and overwrites the slots it reads, so calls
//     that overlap on the GPU (different streams, threads or contexts of one
//     process) race; serialise them;
//   * the success path calls no cudaMalloc, cudaFree or other allocating
//     routine; a rejected call records its message in the context's error text.
#include <mutex>

#include "hydro_f64.cuh"

namespace bsn {
namespace noalloc {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 8;
constexpr long long kCellsPerBlock = (long long)kThreads * kCellsPerThread;   // 2048
constexpr int kMaxPartials = 65536;
constexpr long long kMaxCells = kCellsPerBlock * kMaxPartials;                // 512^3
// A partial that saw a NaN speed holds this pattern; as an unsigned integer it
// is larger than the bits of every non-negative double, Inf included.
constexpr unsigned long long kNaNMark = 0xFFF8000000000000ull;

// Partial maxima (as bit patterns of non-negative doubles) plus one result slot.
static __device__ __align__(256) unsigned long long g_cfl_scratch[kMaxPartials + 32];

__global__ void __launch_bounds__(kThreads) cfl_partial_kernel(const double* U, int nx, int ny, int nz, double g,
                                                               double gm1, double idx, double idy, double idz,
                                                               unsigned long long* partial) {
    Geom G(nx, ny, nz);
    const long long n = (long long)nx * ny * nz;
    const long long first = (long long)blockIdx.x * kCellsPerBlock;
    double m = 0.0;
    bool saw_nan = false;
    for (int r = 0; r < kCellsPerThread; ++r) {
        long long t = first + (long long)r * kThreads + threadIdx.x;
        if (t >= n) break;
        int a = (int)(t % nx); long long q = t / nx; int b = (int)(q % ny); int c = (int)(q / ny);
        long long o = G.act(a, b, c);
        double s = f64::cfl_speed(U[o], U[o + 1], U[o + 2], U[o + 3], U[o + 4], g, gm1, idx, idy, idz);
        if (s != s) saw_nan = true;
        else m = fmax(m, s);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    saw_nan = __any_sync(0xffffffffu, saw_nan);
    __shared__ double wmax[kThreads / 32];
    __shared__ int wnan[kThreads / 32];
    if ((threadIdx.x & 31) == 0) { wmax[threadIdx.x >> 5] = m; wnan[threadIdx.x >> 5] = saw_nan; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double mm = 0.0;
        int nn = 0;
        for (int w = 0; w < kThreads / 32; ++w) { mm = fmax(mm, wmax[w]); nn |= wnan[w]; }
        partial[blockIdx.x] = nn ? kNaNMark : (unsigned long long)__double_as_longlong(mm);
    }
}

__global__ void cfl_final_kernel(unsigned long long* partial, int nblocks, unsigned long long* result) {
    unsigned long long m = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) m = partial[b] > m ? partial[b] : m;
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long other = __shfl_xor_sync(0xffffffffu, m, o);
        m = other > m ? other : m;
    }
    __shared__ unsigned long long wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long r = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = wm[w] > r ? wm[w] : r;
        *result = r;
    }
}

// Device address of g_cfl_scratch, looked up once per device.
std::mutex g_setup_mutex;
unsigned long long* g_scratch_ptr[64] = {nullptr};

// The array of the context's device.  cudaGetSymbolAddress answers for the
// current device, so the current device must be the context's.
bsn_status scratch_for_context_device(bsn_ctx* ctx, unsigned long long** out) {
    int dev = -1;
    BSN_TRY(cuda_check(ctx, cudaGetDevice(&dev), "cudaGetDevice"));
    if (dev != ctx->device)
        return set_err(ctx, BSN_ERR_ARG,
                       "bsn_cfl_dt_3d_f64_noalloc: current device %d is not the context's device %d; make the "
                       "context's device current first",
                       dev, ctx->device);
    if (dev < 0 || dev >= 64) return set_err(ctx, BSN_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        BSN_TRY(cuda_check(ctx, cudaGetSymbolAddress(&p, g_cfl_scratch), "cudaGetSymbolAddress(g_cfl_scratch)"));
        g_scratch_ptr[dev] = (unsigned long long*)p;
    }
    *out = g_scratch_ptr[dev];
    return BSN_OK;
}

}  // namespace noalloc
}  // namespace bsn

using namespace bsn;
using namespace bsn::noalloc;

extern "C" bsn_status bsn_cfl_dt_3d_f64_noalloc(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx,
                                                double dy, double dz, double gamma, double cfl, double* dt_out) {
    if (!ctx) return BSN_ERR_ARG;
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || !dt_out) return set_err(ctx, BSN_ERR_ARG, "U and dt_out must be non-null");
    const long long n = (long long)nx * ny * nz;
    if (n > kMaxCells)
        return set_err(ctx, BSN_ERR_UNSUPPORTED,
                       "bsn_cfl_dt_3d_f64_noalloc: %lld active cells exceed the fixed scratch capacity of %lld "
                       "cells (512^3); use bsn_cfl_dt_3d_f64",
                       n, kMaxCells);
    unsigned long long* scratch = nullptr;
    BSN_TRY(scratch_for_context_device(ctx, &scratch));
    const int nblocks = (int)((n + kCellsPerBlock - 1) / kCellsPerBlock);
    // every partial slot [0, nblocks) and the result slot are written before
    // they are read in this call, so nothing needs clearing
    unsigned long long* result = scratch + kMaxPartials;
    cfl_partial_kernel<<<nblocks, kThreads, 0, ctx->stream>>>(U, nx, ny, nz, gamma, gamma - 1.0, 1.0 / dx, 1.0 / dy,
                                                              1.0 / dz, scratch);
    BSN_TRY(launch_check(ctx, "cfl_partial_kernel"));
    cfl_final_kernel<<<1, 1024, 0, ctx->stream>>>(scratch, nblocks, result);
    BSN_TRY(launch_check(ctx, "cfl_final_kernel"));
    unsigned long long bits = 0;
    BSN_TRY(cuda_check(ctx, cudaMemcpyAsync(&bits, result, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream),
                       "cudaMemcpyAsync(result)"));
    BSN_TRY(cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"));
    if (bits == kNaNMark) {   // as the reference: maximum() is NaN and `NaN > 0.0` is false
        *dt_out = INFINITY;
        return BSN_OK;
    }
    double smax;
    memcpy(&smax, &bits, sizeof(smax));
    *dt_out = smax > 0.0 ? cfl / smax : INFINITY;
    return BSN_OK;
}
