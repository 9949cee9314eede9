// bsn_internal.cuh -- shared device/host plumbing for libbsn (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <map>
#include <set>
#include <tuple>
#include <string>
#include <vector>

#include "bsn.h"

#define BSN_NG 3

// ---------------------------------------------------------------------------
// Context: stream, error text, launch counter and a slot-based workspace that
// grows on demand and is reused across calls (freed by bsn_ctx_destroy).
struct bsn_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    long long launches = 0;
    std::vector<void*> slot_ptr;
    std::vector<size_t> slot_bytes;
    void* pinned = nullptr;          // small pinned host buffer for scalar results
    size_t pinned_bytes = 0;
    void* fft_state = nullptr;       // poisson.cu plan/twiddle cache
    void* fft32_state = nullptr;     // poisson_f32.cu FP32 twiddles and Khat
    // per-kernel CUDA-event timing (bsn_ctx_set_profiling)
    bool profiling = false;
    cudaEvent_t pending_start = nullptr;
    struct Rec { std::string name; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    // stage-kernel tile choice per (precision, driver class, nx, ny, nz):
    // autotuned or forced; tile_last: the latest choice per (precision, nx, ny, nz)
    std::map<std::tuple<int, int, int, int, int>, int> tile_choice;
    std::map<std::tuple<int, int, int, int>, int> tile_last;
    // re-timing pass of a device loop (tile_retime, autotune.cu): the driver
    // class whose choices are re-timed (-1: none), the grids re-timed so far,
    // and the (driver class, precision) pairs whose choices are settled
    int retime_class = -1;
    std::set<std::tuple<int, int, int, int, int>> retimed;
    std::set<std::pair<int, int>> settled;
    int forced_tile[3] = {-1, -1, -1};
    void* learned_state = nullptr;   // learned.cu: packed network parameters
    // graph-captured device time loop (run_steps.cu)
    void* run_state = nullptr;
    void* fmr_run_state = nullptr;   // fmr_f64.cu: graph of the device-resident FMR step
    void* fmrN_state = nullptr;      // fmr_nlevel.cu: nested-level buffers and step graph
    void* coupled_run_state = nullptr;   // coupled_run.cu: graph of the device-resident coupled step
    void* coupled_nested_state = nullptr;   // coupled_run.cu: the coupled step on nested levels
    void* relax_state = nullptr;     // relax.cu: graph of the device-resident relaxation step
    // TMA staging of the stage kernels (tma_host.cu): on unless switched off
    // with bsn_ctx_set_tma; tma_err is the device word a timed-out copy wait sets
    int tma_on = 1;
    unsigned int* tma_err = nullptr;
    int tma_now = 0;                 // the launch being made may use TMA staging (autotune.cu)
    int stiff_guard = 0;             // uniform-grid FP32 steps: stiff faces in FP64 (bsn_ctx_set_stiff_guard)
    int tma_used_last = 0;           // the last stage launch used it
    void* ckpt_state = nullptr;      // h5io.cu: asynchronous checkpoint buffers and writer thread
};

namespace bsn {

enum Slot {
    SLOT_A = 0, SLOT_B, SLOT_UN, SLOT_RED, SLOT_FFT0, SLOT_FFT1, SLOT_PHI, SLOT_RHO,
    SLOT_FMR_UCN, SLOT_FMR_UCNP1, SLOT_FMR_GH, SLOT_FMR_FA, SLOT_FMR_FB, SLOT_FMR_REG,
    SLOT_FMR_BF, SLOT_PHI2, SLOT_RUN, SLOT_FMR_RUN, SLOT_CRUN, SLOT_CRED, SLOT_DIAG, SLOT_DIAGREC, SLOT_RELAX,
    SLOT_SPLIT,
    SLOT_COUNT
};

bsn_status set_err(bsn_ctx* ctx, bsn_status code, const char* fmt, ...);
bsn_status cuda_check(bsn_ctx* ctx, cudaError_t e, const char* what);
bsn_status launch_check(bsn_ctx* ctx, const char* what);
// Record a start event before a launch when profiling is on; launch_check
// records the matching stop event.
void prof_begin(bsn_ctx* ctx);
void* slot(bsn_ctx* ctx, int s, size_t bytes, bsn_status* st);
void* pinned(bsn_ctx* ctx, size_t bytes, bsn_status* st);
namespace tma {
void init_ctx(bsn_ctx* ctx);             // tma_host.cu: error word of the context's device
bsn_status check_error(bsn_ctx* ctx);    // BSN_ERR_TIMEOUT if a staging copy wait ran out (synchronises)
}  // namespace tma

#define BSN_TRY(expr)                         \
    do {                                      \
        bsn_status _s = (expr);               \
        if (_s != BSN_OK) return _s;          \
    } while (0)

#define BSN_CUDA(ctx, expr) BSN_TRY(::bsn::cuda_check((ctx), (expr), #expr))

// ---------------------------------------------------------------------------
// Julia Base semantics for Float64 max/min/clamp (NaN propagates; max(+0,-0)
// = +0, min(+0,-0) = -0; clamp(x,lo,hi) = x>hi ? hi : x<lo ? lo : x).
template <typename T>
__host__ __device__ __forceinline__ T jmax(T x, T y) {
    if (x != x || y != y) return x + y;
    if (x > y) return x;
    if (y > x) return y;
    return signbit(x) ? y : x;
}
template <typename T>
__host__ __device__ __forceinline__ T jmin(T x, T y) {
    if (x != x || y != y) return x + y;
    if (x < y) return x;
    if (y < x) return y;
    return signbit(x) ? x : y;
}
template <typename T>
__host__ __device__ __forceinline__ T jclamp(T x, T lo, T hi) {
    return x > hi ? hi : (x < lo ? lo : x);
}
template <typename T>
__host__ __device__ __forceinline__ T sq(T x) { return x * x; }

// Geometry of a ghosted state array U[q,i,j,k].
struct Geom {
    int nx, ny, nz;
    long long sy, sz;   // element strides of j and k (q stride 1, i stride 5)
    __host__ __device__ Geom() {}
    __host__ __device__ Geom(int a, int b, int c)
        : nx(a), ny(b), nz(c), sy(5LL * (a + 2 * BSN_NG)), sz(5LL * (a + 2 * BSN_NG) * (b + 2 * BSN_NG)) {}
    // 0-based GHOSTED indices
    __host__ __device__ long long at(int i, int j, int k) const { return 5LL * i + sy * j + sz * k; }
    // 0-based ACTIVE indices
    __host__ __device__ long long act(int a, int b, int c) const {
        return at(a + BSN_NG, b + BSN_NG, c + BSN_NG);
    }
    __host__ __device__ long long ncell() const {
        return (long long)(nx + 2 * BSN_NG) * (ny + 2 * BSN_NG) * (nz + 2 * BSN_NG);
    }
    __host__ __device__ long long nelem() const { return 5LL * ncell(); }
};

// Ghost-source mapping of a position along one axis (active-relative, may be
// in [-3, n+3)): the active cell a ghost copies under outflow/periodic BCs.
// Composes the reference's x->y->z fill order (src/euler3d.jl:33-62) per axis.
__host__ __device__ __forceinline__ int bc_map(int a, int n, int bc) {
    if (a >= 0 && a < n) return a;
    if (bc == BSN_BC_PERIODIC) {
        int m = a % n;
        return m < 0 ? m + n : m;
    }
    return a < 0 ? 0 : n - 1;
}

inline unsigned grid1d(long long n, int block) {
    long long g = (n + block - 1) / block;
    return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace bsn
