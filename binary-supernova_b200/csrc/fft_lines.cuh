// fft_lines.cuh -- the batched FFT passes of the isolated Poisson solve,
// templated on the complex type: double2 for the FP64 path (poisson.cu) and
// float2 for the FP32 path (poisson_f32.cu).  Inputs (the density) and the
// output potential stay FP64 in HBM; the transforms and the spectrum run in
// the complex type.
//
// Each line of N = 2^LOGN points is transformed by T = N / E threads that hold
// E = min(N, 16) points each in registers: a self-sorting (Stockham) FFT of
// radix-16 passes and one smaller last pass where LOGN is not a multiple of 4
// (Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC 2008).  A pass's radix-R butterflies run in
// registers; the passes exchange through shared memory, so a 256-point line
// (the 128^3 grid padded to 256) makes one shared-memory round trip and two
// barriers where a radix-2 transform in shared memory makes eight.  The first
// pass reads, and the last pass writes, HBM directly: thread t holds elements
// t + k*T of its line, in natural order in and out, so neighbouring threads
// touch neighbouring addresses on the contiguous axis and line batches of
// neighbouring kx coalesce on the strided ones.  Twiddles exp(-2 pi i k / N)
// come from a table built in long double on the host (k < N/2; the other half
// by symmetry); the radix-16 butterflies use the exact values of cos(pi k / 8).
//
// The Green's-function transform (built once per grid, poisson.cu) keeps the
// radix-2 transform in shared memory below (fft_dit).
#pragma once

#include "bsn_internal.cuh"

namespace bsn {
namespace fft {

template <class C> struct Cx;
template <> struct Cx<double2> {
    using R = double;
    static __host__ __device__ double2 mk(double a, double b) { return make_double2(a, b); }
};
template <> struct Cx<float2> {
    using R = float;
    static __host__ __device__ float2 mk(float a, float b) { return make_float2(a, b); }
};

// complex product with the two sums as fused multiply-adds (the FP64 solve's
// translation unit is built without contraction; the transforms are not
// bound to the oracle's rounding, only to its tolerance)
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -(a.y * b.y)), fmaf(a.x, b.y, a.y * b.x));
}

__device__ __forceinline__ int bitrev(int v, int logn) { return (int)(__brev((unsigned)v) >> (32 - logn)); }

template <class C>
__device__ void fft_dit(C* s, const C* tw, int lines, int logn, bool inverse) {
    const int N = 1 << logn, H = N >> 1;
    for (int half = 1, lh = 0; half < N; half <<= 1, ++lh) {
        __syncthreads();
        for (int b = threadIdx.x; b < lines * H; b += blockDim.x) {
            int l = b >> (logn - 1), j = b & (H - 1);
            int grp = j >> lh, pos = j & (half - 1);
            int i0 = l * N + (grp << (lh + 1)) + pos, i1 = i0 + half;
            C w = tw[pos << (logn - 1 - lh)];
            if (inverse) w.y = -w.y;
            C a = s[i0], c = cmul(w, s[i1]);
            s[i0] = Cx<C>::mk(a.x + c.x, a.y + c.y);
            s[i1] = Cx<C>::mk(a.x - c.x, a.y - c.y);
        }
    }
    __syncthreads();
}

template <class C>
__device__ void load_twiddles(C* stw, const C* tw, int logn) {
    for (int t = threadIdx.x; t < (1 << (logn - 1)); t += blockDim.x) stw[t] = tw[t];
}

// Density source: rho array (nx,ny,nz) or the state U (q = 0), optionally
// floored as euler3d_rhs! floors before the source is added.
struct RhoSrc {
    const double* rho;
    const double* U;
    int nx, ny, nz;
    double rho_floor;   // < 0: no floor
    __device__ double at(int x, int y, int z) const {
        double r;
        if (rho) r = rho[x + (long long)nx * (y + (long long)ny * z)];
        else {
            long long X = nx + 2 * BSN_NG, Y = ny + 2 * BSN_NG;
            r = U[5LL * ((x + BSN_NG) + X * ((y + BSN_NG) + Y * (long long)(z + BSN_NG)))];
        }
        if (rho_floor >= 0.0 && r < rho_floor) r = rho_floor;
        return r;
    }
};


// ---- register-resident line FFT ---------------------------------------------

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }
__host__ __device__ constexpr int brevc(int v, int bits) {
    int r = 0;
    for (int i = 0; i < bits; ++i)
        if ((v >> i) & 1) r |= 1 << (bits - 1 - i);
    return r;
}

// Shape of the transform of one line of N = 2^LOGN points.
template <int LOGN>
struct LineShape {
    static_assert(LOGN >= 1 && LOGN <= 12, "line FFT length 2..4096");
    static constexpr int N = 1 << LOGN;
    static constexpr int E = N < 16 ? N : 16;          // points per thread
    static constexpr int T = N / E;                      // threads per line
    static constexpr int NP = LOGN <= 4 ? 1 : (LOGN + 3) / 4;   // passes
    __host__ __device__ static constexpr int log_radix(int p) { return LOGN <= 4 ? LOGN : (p < LOGN / 4 ? 4 : LOGN % 4); }
    __host__ __device__ static constexpr int log_span(int p) { return p == 0 ? 0 : log_span(p - 1) + log_radix(p - 1); }
    static constexpr int PAD = N + N / 16;               // padded row length (line-major exchange)
};

template <class C>
__device__ __forceinline__ C cadd(C a, C b) { return Cx<C>::mk(a.x + b.x, a.y + b.y); }
template <class C>
__device__ __forceinline__ C csub(C a, C b) { return Cx<C>::mk(a.x - b.x, a.y - b.y); }

// a * w, or a * conj(w) for the inverse transform
template <class C, bool INV>
__device__ __forceinline__ C twmul(C a, C w) {
    if (INV) w.y = -w.y;
    return cmul(a, w);
}

// a * exp(-+2 pi i k / 16), k < 8 (compile-time after unrolling)
template <class C, bool INV>
__device__ __forceinline__ C mul_w16(C a, int k) {
    using R = typename Cx<C>::R;
    constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173, h = 0.70710678118654752440;
    if (k == 0) return a;
    if (k == 4) return INV ? Cx<C>::mk(-a.y, a.x) : Cx<C>::mk(a.y, -a.x);
    double wr, wi;
    switch (k) {
        case 1: wr = c1; wi = -s1; break;
        case 2: wr = h; wi = -h; break;
        case 3: wr = s1; wi = -c1; break;
        case 5: wr = -s1; wi = -c1; break;
        case 6: wr = -h; wi = -h; break;
        default: wr = -c1; wi = -s1; break;
    }
    return twmul<C, INV>(a, Cx<C>::mk((R)wr, (R)wi));
}

// In-register DFT of R = 2, 4, 8 or 16 points, natural order in and out
// (radix-2 decimation in time over a compile-time bit reversal).
template <class C, int R, bool INV>
__device__ __forceinline__ void dft(C (&a)[R]) {
    constexpr int LR = ilog2c(R);
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int j = brevc(i, LR);
        if (j > i) { C t = a[i]; a[i] = a[j]; a[j] = t; }
    }
#pragma unroll
    for (int half = 1; half < R; half <<= 1) {
#pragma unroll
        for (int i = 0; i < R; i += 2 * half) {
#pragma unroll
            for (int p = 0; p < half; ++p) {
                C b = mul_w16<C, INV>(a[i + p + half], p * (16 / (2 * half)));
                C x = a[i + p];
                a[i + p] = cadd(x, b);
                a[i + p + half] = csub(x, b);
            }
        }
    }
}

// exp(-2 pi i k / N) for k < N from the table of k < N/2
template <class C>
__device__ __forceinline__ C twiddle(const C* tw, int k, int N) {
    if (k < (N >> 1)) return tw[k];
    C w = tw[k - (N >> 1)];
    return Cx<C>::mk(-w.x, -w.y);
}

// Shared-memory layouts of the exchange between passes: a line's points in a
// padded row (lines along the contiguous axis: the T threads of a line are
// neighbours), or point-major with the batch's lines innermost (lines along a
// strided axis: neighbouring threads hold neighbouring lines).
template <int LOGN>
struct RowLayout {
    __device__ __forceinline__ int at(int l, int i) const { return l * LineShape<LOGN>::PAD + i + (i >> 4); }
};
struct ColLayout {
    int L;
    __device__ __forceinline__ int at(int l, int i) const { return i * L + l; }
};

// Pass P of the Stockham FFT of line l; v holds points t + k*T on entry to
// pass 0 and the transform's points t + k*T after the last pass.  Every
// thread of the block calls it (barriers inside).
template <class C, int LOGN, bool INV, int P, class Lay>
__device__ __forceinline__ void fft_pass(C (&v)[LineShape<LOGN>::E], C* S, const Lay& lay, int l, int t,
                                         const C* tw) {
    using Sh = LineShape<LOGN>;
    constexpr int N = Sh::N, E = Sh::E, T = Sh::T;
    constexpr int R = 1 << Sh::log_radix(P), NS = 1 << Sh::log_span(P), M = E / R;
    constexpr bool LAST = P == Sh::NP - 1;
    C a[E];
    if constexpr (P == 0) {
#pragma unroll
        for (int m = 0; m < M; ++m)
#pragma unroll
            for (int r = 0; r < R; ++r) a[m * R + r] = v[m + r * M];
    } else {
#pragma unroll
        for (int m = 0; m < M; ++m)
#pragma unroll
            for (int r = 0; r < R; ++r) a[m * R + r] = S[lay.at(l, t + m * T + r * (N / R))];
        __syncthreads();   // every read of this pass is done before the writes below
    }
#pragma unroll
    for (int m = 0; m < M; ++m) {
        C b[R];
        const int jm = (t + m * T) & (NS - 1);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            b[r] = a[m * R + r];
            if (NS > 1 && r > 0) b[r] = twmul<C, INV>(b[r], twiddle(tw, jm * r * (N / (NS * R)), N));
        }
        dft<C, R, INV>(b);
#pragma unroll
        for (int r = 0; r < R; ++r) a[m * R + r] = b[r];
    }
    if constexpr (LAST) {
#pragma unroll
        for (int m = 0; m < M; ++m)
#pragma unroll
            for (int r = 0; r < R; ++r) v[m + r * M] = a[m * R + r];
    } else {
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const int j = t + m * T;
            const int d = (j / NS) * NS * R + (j & (NS - 1));
#pragma unroll
            for (int r = 0; r < R; ++r) S[lay.at(l, d + r * NS)] = a[m * R + r];
        }
        __syncthreads();
        fft_pass<C, LOGN, INV, P + 1>(v, S, lay, l, t, tw);
    }
}

template <class C, int LOGN, bool INV, class Lay>
__device__ __forceinline__ void line_fft(C (&v)[LineShape<LOGN>::E], C* S, const Lay& lay, int l, int t,
                                         const C* tw) {
    fft_pass<C, LOGN, INV, 0>(v, S, lay, l, t, tw);
}

// Pass 1: x forward over the ny*nz rows holding density (rows are lines);
// W1[kx + (nx+1)*(y + ny*z)], kx <= nx.  A block is `lines` rows x T threads.
template <class C, int LOGN>
__global__ void __launch_bounds__(256) fwd_x_kernel(RhoSrc src, C* W1, const C* tw, int lines) {
    using Sh = LineShape<LOGN>;
    using R = typename Cx<C>::R;
    constexpr int E = Sh::E, T = Sh::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw);
    const int t = threadIdx.x % T, l = threadIdx.x / T, nx = src.nx;
    const long long nrows = (long long)src.ny * src.nz;
    const long long row = (long long)blockIdx.x * lines + l;
    const bool ok = row < nrows;
    const int y = ok ? (int)(row % src.ny) : 0, z = ok ? (int)(row / src.ny) : 0;
    C v[E];
#pragma unroll
    for (int k = 0; k < E; ++k)   // points t + k*T < N/2 = nx hold density, the rest is padding
        v[k] = Cx<C>::mk((ok && k < E / 2) ? (R)src.at(t + k * T, y, z) : R(0), R(0));
    line_fft<C, LOGN, false>(v, S, RowLayout<LOGN>{}, l, t, tw);
    if (!ok) return;
    C* out = W1 + (long long)(nx + 1) * row;
#pragma unroll
    for (int k = 0; k <= E / 2; ++k) {
        const int kx = t + k * T;
        if (kx <= nx) out[kx] = v[k];
    }
}

// Generic strided-line pass over a complex array: lines run along an axis of
// stride `estride`; a block takes `lines` neighbouring lines (stride 1, the kx
// axis, length nkx) at a fixed outer index.  Input samples t < n_in are read
// (the rest are zero); outputs t < n_out are written.
template <class C>
struct AxisIO {
    const C* in;
    C* out;
    int nkx;              // extent of the contiguous (line-batch) axis
    long long nouter;     // number of outer positions
    long long in_estride, out_estride;   // element stride along the line
    long long in_ostride, out_ostride;   // stride of the outer index
    int n_in, n_out;
};

template <class C, int LOGN, bool INV>
__global__ void __launch_bounds__(256) axis_kernel(AxisIO<C> io, const C* tw, int lines) {
    using Sh = LineShape<LOGN>;
    using R = typename Cx<C>::R;
    constexpr int E = Sh::E, T = Sh::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw);
    const int l = threadIdx.x % lines, t = threadIdx.x / lines;
    const int nbx = (io.nkx + lines - 1) / lines;
    const long long outer = blockIdx.x / nbx;
    const int kx = (int)(blockIdx.x % nbx) * lines + l;
    const bool ok = kx < io.nkx;
    const C* in = io.in + kx + outer * io.in_ostride;
    C v[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int e = t + k * T;
        v[k] = (ok && e < io.n_in) ? in[e * io.in_estride] : Cx<C>::mk(R(0), R(0));
    }
    line_fft<C, LOGN, INV>(v, S, ColLayout{lines}, l, t, tw);
    if (!ok) return;
    C* out = io.out + kx + outer * io.out_ostride;
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int e = t + k * T;
        if (e < io.n_out) out[e * io.out_estride] = v[k];
    }
}

// z forward * Khat * z inverse per line, in place in
// W2[kx + (nx+1)*(kyl + nky*z)] for ky = ky0 + kyl (the whole ky range
// ky0 = 0, nky = N2 on one GPU; a rank's share of it after the transpose of
// a z-slab decomposition), z < nz in and out.
template <class C, int LOGN>
__global__ void __launch_bounds__(256, 2) z_conv_kernel(C* W2, const typename Cx<C>::R* khat, int nx, int N2, int ny,
                                                     int nz, int lines, const C* tw, int ky0, int nky) {
    using Sh = LineShape<LOGN>;
    using R = typename Cx<C>::R;
    constexpr int N = Sh::N, E = Sh::E, T = Sh::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw);
    const int l = threadIdx.x % lines, t = threadIdx.x / lines;
    const int nkx = nx + 1;
    const int nbx = (nkx + lines - 1) / lines;
    const int kyl = blockIdx.x / nbx, ky = ky0 + kyl;
    const int kx = (int)(blockIdx.x % nbx) * lines + l;
    const bool ok = kx < nkx;
    const long long plane = (long long)nkx * nky;
    C* line = W2 + kx + (long long)nkx * kyl;
    C v[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {   // z = t + k*T < N/2 = nz hold data
        v[k] = (ok && k < E / 2) ? line[plane * (t + k * T)] : Cx<C>::mk(R(0), R(0));
    }
    line_fft<C, LOGN, false>(v, S, ColLayout{lines}, l, t, tw);
    const int kyf = ky <= ny ? ky : N2 - ky;
    const R* kh = khat + (ok ? kx : 0) + (long long)nkx * kyf;
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int kz = t + k * T;
        const int kzf = kz <= nz ? kz : N - kz;
        const R g = kh[(long long)nkx * (ny + 1) * kzf];
        v[k] = Cx<C>::mk(v[k].x * g, v[k].y * g);
    }
    line_fft<C, LOGN, true>(v, S, ColLayout{lines}, l, t, tw);
    if (!ok) return;
#pragma unroll
    for (int k = 0; k < E / 2; ++k) line[plane * (t + k * T)] = v[k];
}

// x inverse of the Hermitian rows W1[kx <= nx] -> real Phi[x < nx] (FP64).
template <class C, int LOGN>
__global__ void __launch_bounds__(256) inv_x_kernel(const C* W1, double* phi, int nx, int ny, int nz, int lines,
                                                    const C* tw) {
    using Sh = LineShape<LOGN>;
    using R = typename Cx<C>::R;
    constexpr int N = Sh::N, E = Sh::E, T = Sh::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw);
    const int t = threadIdx.x % T, l = threadIdx.x / T;
    const long long nrows = (long long)ny * nz;
    const long long row = (long long)blockIdx.x * lines + l;
    const bool ok = row < nrows;
    const C* in = W1 + (long long)(nx + 1) * (ok ? row : 0);
    C v[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int i = t + k * T;
        C c = Cx<C>::mk(R(0), R(0));
        if (ok) {
            if (i <= nx) c = in[i];
            else { c = in[N - i]; c.y = -c.y; }
        }
        v[k] = c;
    }
    line_fft<C, LOGN, true>(v, S, RowLayout<LOGN>{}, l, t, tw);
    if (!ok) return;
    double* out = phi + (long long)nx * row;
#pragma unroll
    for (int k = 0; k < E / 2; ++k) out[t + k * T] = (double)v[k].x;
}

// ---- host side ----------------------------------------------------------------

inline int fft_ilog2(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

// Launch geometry of a pass of length 2^LOGN: rows (contiguous lines) or kx
// lines (strided lines) per block, block size and dynamic shared memory.
template <int LOGN>
struct PassGeom {
    using Sh = LineShape<LOGN>;
    static constexpr int row_lines = Sh::T >= 256 ? 1 : 256 / Sh::T;
    static constexpr int col_lines = Sh::T <= 16 ? 16 : (Sh::T >= 256 ? 1 : 256 / Sh::T);
    template <class C> static size_t row_smem() { return sizeof(C) * (size_t)row_lines * Sh::PAD; }
    template <class C> static size_t col_smem() { return sizeof(C) * (size_t)col_lines * Sh::N; }
};

// Opt a kernel into its dynamic shared memory once per device.
inline bsn_status smem_optin(bsn_ctx* ctx, const void* fn, size_t bytes, bool* done) {
    const int dev = ctx->device & 63;
    if (!done[dev]) {
        BSN_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        done[dev] = true;
    }
    return BSN_OK;
}

template <class C, int LOGN>
bsn_status launch_fwd_x(bsn_ctx* ctx, const RhoSrc& src, C* W1, const C* tw) {
    using G = PassGeom<LOGN>;
    static bool done[64] = {false};
    const size_t sm = G::template row_smem<C>();
    BSN_TRY(smem_optin(ctx, (const void*)fwd_x_kernel<C, LOGN>, sm, done));
    const long long rows = (long long)src.ny * src.nz;
    prof_begin(ctx);
    fwd_x_kernel<C, LOGN><<<grid1d(rows, G::row_lines), G::row_lines * LineShape<LOGN>::T, sm, ctx->stream>>>(
        src, W1, tw, G::row_lines);
    return launch_check(ctx, "fwd_x_kernel");
}

template <class C, int LOGN, bool INV>
bsn_status launch_axis(bsn_ctx* ctx, const AxisIO<C>& io, const C* tw) {
    using G = PassGeom<LOGN>;
    static bool done[64] = {false};
    const size_t sm = G::template col_smem<C>();
    BSN_TRY(smem_optin(ctx, (const void*)axis_kernel<C, LOGN, INV>, sm, done));
    const long long nbx = (io.nkx + G::col_lines - 1) / G::col_lines;
    prof_begin(ctx);
    axis_kernel<C, LOGN, INV><<<(unsigned)(nbx * io.nouter), G::col_lines * LineShape<LOGN>::T, sm, ctx->stream>>>(
        io, tw, G::col_lines);
    return launch_check(ctx, "fft_y_kernel");
}

template <class C, int LOGN>
bsn_status launch_zconv(bsn_ctx* ctx, C* W2, const typename Cx<C>::R* K, const C* tw, int nx, int ny, int nz,
                        int ky0, int nky) {
    using G = PassGeom<LOGN>;
    static bool done[64] = {false};
    const size_t sm = G::template col_smem<C>();
    BSN_TRY(smem_optin(ctx, (const void*)z_conv_kernel<C, LOGN>, sm, done));
    const long long nbx = (nx + 1 + G::col_lines - 1) / G::col_lines;
    prof_begin(ctx);
    z_conv_kernel<C, LOGN><<<(unsigned)(nbx * nky), G::col_lines * LineShape<LOGN>::T, sm, ctx->stream>>>(
        W2, K, nx, 2 * ny, ny, nz, G::col_lines, tw, ky0, nky);
    return launch_check(ctx, "z_conv_kernel");
}

template <class C, int LOGN>
bsn_status launch_inv_x(bsn_ctx* ctx, const C* W1, double* phi, int nx, int ny, int nz, const C* tw) {
    using G = PassGeom<LOGN>;
    static bool done[64] = {false};
    const size_t sm = G::template row_smem<C>();
    BSN_TRY(smem_optin(ctx, (const void*)inv_x_kernel<C, LOGN>, sm, done));
    const long long rows = (long long)ny * nz;
    prof_begin(ctx);
    inv_x_kernel<C, LOGN><<<grid1d(rows, G::row_lines), G::row_lines * LineShape<LOGN>::T, sm, ctx->stream>>>(
        W1, phi, nx, ny, nz, G::row_lines, tw);
    return launch_check(ctx, "inv_x_kernel");
}

// Run F<LOGN>() for the line length 2^logn, 4 <= 2^logn <= 4096.
template <class F>
bsn_status by_length(bsn_ctx* ctx, int logn, F&& f) {
    switch (logn) {
        case 2: return f(std::integral_constant<int, 2>{});
        case 3: return f(std::integral_constant<int, 3>{});
        case 4: return f(std::integral_constant<int, 4>{});
        case 5: return f(std::integral_constant<int, 5>{});
        case 6: return f(std::integral_constant<int, 6>{});
        case 7: return f(std::integral_constant<int, 7>{});
        case 8: return f(std::integral_constant<int, 8>{});
        case 9: return f(std::integral_constant<int, 9>{});
        case 10: return f(std::integral_constant<int, 10>{});
        case 11: return f(std::integral_constant<int, 11>{});
        case 12: return f(std::integral_constant<int, 12>{});
        default: return set_err(ctx, BSN_ERR_UNSUPPORTED, "FFT line length 2^%d outside 4..4096", logn);
    }
}

// The five passes of one solve.  K: Khat (real, (nx+1)(ny+1)(nz+1));
// t1..t3: twiddles of the doubled lengths; W1, W2: workspaces of
// (nx+1) ny nz and (nx+1) N2 nz complex values.
template <class C>
bsn_status fwd_xy(bsn_ctx* ctx, const RhoSrc& src, const C* t1, const C* t2, C* W1, C* W2) {
    const int nx = src.nx, ny = src.ny, nz = src.nz, N2 = 2 * ny;
    BSN_TRY(by_length(ctx, fft_ilog2(2 * nx), [&](auto L) { return launch_fwd_x<C, decltype(L)::value>(ctx, src, W1, t1); }));
    AxisIO<C> y1{W1, W2, nx + 1, nz, nx + 1, nx + 1, (long long)(nx + 1) * ny, (long long)(nx + 1) * N2, ny, N2};
    return by_length(ctx, fft_ilog2(N2), [&](auto L) { return launch_axis<C, decltype(L)::value, false>(ctx, y1, t2); });
}

template <class C>
bsn_status inv_yx(bsn_ctx* ctx, const C* W2, const C* t1, const C* t2, C* W1, double* phi, int nx, int ny, int nz) {
    const int N2 = 2 * ny;
    AxisIO<C> y2{W2, W1, nx + 1, nz, nx + 1, nx + 1, (long long)(nx + 1) * N2, (long long)(nx + 1) * ny, N2, ny};
    BSN_TRY(by_length(ctx, fft_ilog2(N2), [&](auto L) { return launch_axis<C, decltype(L)::value, true>(ctx, y2, t2); }));
    return by_length(ctx, fft_ilog2(2 * nx),
                     [&](auto L) { return launch_inv_x<C, decltype(L)::value>(ctx, W1, phi, nx, ny, nz, t1); });
}

template <class C>
bsn_status solve_lines(bsn_ctx* ctx, const RhoSrc& src, const typename Cx<C>::R* K, const C* t1, const C* t2,
                       const C* t3, C* W1, C* W2, double* phi) {
    const int nx = src.nx, ny = src.ny, nz = src.nz;
    BSN_TRY(fwd_xy<C>(ctx, src, t1, t2, W1, W2));
    BSN_TRY(by_length(ctx, fft_ilog2(2 * nz),
                      [&](auto L) { return launch_zconv<C, decltype(L)::value>(ctx, W2, K, t3, nx, ny, nz, 0, 2 * ny); }));
    return inv_yx<C>(ctx, W2, t1, t2, W1, phi, nx, ny, nz);
}

// The solve split at the z transform, for a z-slab decomposition (one rank
// per slab of nzl planes; the kernels and their per-line arithmetic are those
// of solve_lines, so the assembled potential is bit-identical to it).
// Forward: x and y transforms of the slab's nzl density planes into
// W2[kx + (nx+1)*(ky + N2*z)], z < nzl (W1: (nx+1) ny nzl scratch).
template <class C>
bsn_status slab_forward_lines(bsn_ctx* ctx, const RhoSrc& src, const C* t1, const C* t2, C* W1, C* W2) {
    return fwd_xy<C>(ctx, src, t1, t2, W1, W2);
}

// z lines of the global grid (nz planes) for ky in [ky0, ky0 + nky), in place
// in T[kx + (nx+1)*(kyl + nky*z)].
template <class C>
bsn_status slab_zconv_lines(bsn_ctx* ctx, C* T, const typename Cx<C>::R* K, const C* t3, int nx, int ny, int nz,
                            int ky0, int nky) {
    if (nky < 1) return BSN_OK;
    return by_length(ctx, fft_ilog2(2 * nz),
                     [&](auto L) { return launch_zconv<C, decltype(L)::value>(ctx, T, K, t3, nx, ny, nz, ky0, nky); });
}

// Inverse: y and x transforms of the slab's W2 (z < nzl) into its nzl planes
// of Phi (W1: (nx+1) ny nzl scratch; W2 is left as it was).
template <class C>
bsn_status slab_inverse_lines(bsn_ctx* ctx, const C* W2, const C* t1, const C* t2, C* W1, double* phi, int nx,
                              int ny, int nz) {
    return inv_yx<C>(ctx, W2, t1, t2, W1, phi, nx, ny, nz);
}

}  // namespace fft
}  // namespace bsn
