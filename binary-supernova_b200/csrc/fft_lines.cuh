// fft_lines.cuh -- the batched in-shared-memory FFT passes of the isolated
// Poisson solve, templated on the complex type: double2 for the FP64 path
// (poisson.cu) and float2 for the FP32 path (poisson_f32.cu).  Inputs (the
// density) and the output potential stay FP64 in HBM; the transforms and the
// spectrum run in the complex type.
//
// Every transform is a radix-2 FFT over a batch of `lines` lines of length
// N = 2^logn held in shared memory (twiddles exp(-2 pi i t / N), t < N/2,
// staged first); DIT takes bit-reversed input to natural order, DIF natural
// to bit-reversed.  Line batches are chosen so neighbouring elements are
// contiguous in HBM: loads and stores coalesce on all three axes.
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

template <class C>
__device__ __forceinline__ C cmul(C a, C b) {
    return Cx<C>::mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
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
__device__ void fft_dif(C* s, const C* tw, int lines, int logn, bool inverse) {
    const int N = 1 << logn, H = N >> 1;
    for (int half = H, lh = logn - 1; half >= 1; half >>= 1, --lh) {
        __syncthreads();
        for (int b = threadIdx.x; b < lines * H; b += blockDim.x) {
            int l = b >> (logn - 1), j = b & (H - 1);
            int grp = j >> lh, pos = j & (half - 1);
            int i0 = l * N + (grp << (lh + 1)) + pos, i1 = i0 + half;
            C w = tw[pos << (logn - 1 - lh)];
            if (inverse) w.y = -w.y;
            C a = s[i0], c = s[i1];
            s[i0] = Cx<C>::mk(a.x + c.x, a.y + c.y);
            s[i1] = cmul(w, Cx<C>::mk(a.x - c.x, a.y - c.y));
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

// Pass 1: x-forward over the ny*nz rows holding density (rows are lines).
// W1[kx + (nx+1)*(y + ny*z)], kx <= nx.
template <class C>
__global__ void fwd_x_kernel(RhoSrc src, C* W1, const C* tw, int logn, int lines) {
    using R = typename Cx<C>::R;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int N = 1 << logn, nx = src.nx;
    C* stw = sm;
    C* s = sm + (N >> 1);
    load_twiddles(stw, tw, logn);
    long long nrows = (long long)src.ny * src.nz;
    long long row0 = (long long)blockIdx.x * lines;
    for (int t = threadIdx.x; t < lines * N; t += blockDim.x) s[t] = Cx<C>::mk(R(0), R(0));
    __syncthreads();
    for (int t = threadIdx.x; t < lines * nx; t += blockDim.x) {
        int l = t / nx, x = t - l * nx;
        long long row = row0 + l;
        if (row >= nrows) continue;
        int y = (int)(row % src.ny), z = (int)(row / src.ny);
        s[l * N + bitrev(x, logn)] = Cx<C>::mk((R)src.at(x, y, z), R(0));
    }
    fft_dit(s, stw, lines, logn, false);
    for (int t = threadIdx.x; t < lines * (nx + 1); t += blockDim.x) {
        int l = t / (nx + 1), kx = t - l * (nx + 1);
        long long row = row0 + l;
        if (row >= nrows) continue;
        W1[kx + (long long)(nx + 1) * row] = s[l * N + kx];
    }
}

// Generic strided-line pass over a complex array: lines run along an axis of
// stride `estride`; a CTA takes `lines` neighbouring lines (stride 1, the kx
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

template <class C>
__global__ void axis_kernel(AxisIO<C> io, const C* tw, int logn, int lines, int inverse) {
    using R = typename Cx<C>::R;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int N = 1 << logn;
    C* stw = sm;
    C* s = sm + (N >> 1);
    load_twiddles(stw, tw, logn);
    int nbx = (io.nkx + lines - 1) / lines;
    long long outer = blockIdx.x / nbx;
    int kx0 = (int)(blockIdx.x % nbx) * lines;
    for (int t = threadIdx.x; t < lines * N; t += blockDim.x) s[t] = Cx<C>::mk(R(0), R(0));
    __syncthreads();
    for (int t = threadIdx.x; t < lines * io.n_in; t += blockDim.x) {
        int l = t % lines, e = t / lines;
        int kx = kx0 + l;
        if (kx >= io.nkx) continue;
        s[l * N + bitrev(e, logn)] = io.in[kx + outer * io.in_ostride + e * io.in_estride];
    }
    fft_dit(s, stw, lines, logn, inverse != 0);
    for (int t = threadIdx.x; t < lines * io.n_out; t += blockDim.x) {
        int l = t % lines, e = t / lines;
        int kx = kx0 + l;
        if (kx >= io.nkx) continue;
        io.out[kx + outer * io.out_ostride + e * io.out_estride] = s[l * N + e];
    }
}

// z forward (DIF) * Khat (bit-reversed order) * z inverse (DIT), in place in
// W2[kx + (nx+1)*(kyl + nky*z)] for ky = ky0 + kyl (the whole ky range
// ky0 = 0, nky = N2 on one GPU; a rank's share of it after the transpose of
// a z-slab decomposition), z < nz in and out.
template <class C>
__global__ void z_conv_kernel(C* W2, const typename Cx<C>::R* khat, int nx, int N2, int ny, int nz, int logn,
                              int lines, const C* tw, int ky0, int nky) {
    using R = typename Cx<C>::R;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int N = 1 << logn;
    C* stw = sm;
    C* s = sm + (N >> 1);
    load_twiddles(stw, tw, logn);
    int nkx = nx + 1;
    int nbx = (nkx + lines - 1) / lines;
    const int kyl = blockIdx.x / nbx, ky = ky0 + kyl;
    int kx0 = (blockIdx.x % nbx) * lines;
    long long plane = (long long)nkx * nky;
    for (int t = threadIdx.x; t < lines * N; t += blockDim.x) s[t] = Cx<C>::mk(R(0), R(0));
    __syncthreads();
    for (int t = threadIdx.x; t < lines * nz; t += blockDim.x) {
        int l = t % lines, z = t / lines;
        int kx = kx0 + l;
        if (kx >= nkx) continue;
        s[l * N + z] = W2[kx + (long long)nkx * kyl + plane * z];
    }
    fft_dif(s, stw, lines, logn, false);
    int kyf = ky <= ny ? ky : N2 - ky;
    for (int t = threadIdx.x; t < lines * N; t += blockDim.x) {
        int l = t / N, p = t - l * N;
        int kx = kx0 + l;
        if (kx >= nkx) continue;
        int kz = bitrev(p, logn);
        int kzf = kz <= nz ? kz : N - kz;
        R k = khat[kx + (long long)nkx * (kyf + (long long)(ny + 1) * kzf)];
        s[t] = Cx<C>::mk(s[t].x * k, s[t].y * k);
    }
    fft_dit(s, stw, lines, logn, true);
    for (int t = threadIdx.x; t < lines * nz; t += blockDim.x) {
        int l = t % lines, z = t / lines;
        int kx = kx0 + l;
        if (kx >= nkx) continue;
        W2[kx + (long long)nkx * kyl + plane * z] = s[l * N + z];
    }
}

// x inverse of the Hermitian rows W1[kx <= nx] -> real Phi[x < nx] (FP64).
template <class C>
__global__ void inv_x_kernel(const C* W1, double* phi, int nx, int ny, int nz, int logn, int lines, const C* tw) {
    using R = typename Cx<C>::R;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int N = 1 << logn;
    C* stw = sm;
    C* s = sm + (N >> 1);
    load_twiddles(stw, tw, logn);
    long long nrows = (long long)ny * nz;
    long long row0 = (long long)blockIdx.x * lines;
    for (int t = threadIdx.x; t < lines * N; t += blockDim.x) {
        int l = t / N, k = t - l * N;
        long long row = row0 + l;
        C v = Cx<C>::mk(R(0), R(0));
        if (row < nrows) {
            if (k <= nx) v = W1[k + (long long)(nx + 1) * row];
            else { C c = W1[(N - k) + (long long)(nx + 1) * row]; v = Cx<C>::mk(c.x, -c.y); }
        }
        s[l * N + bitrev(k, logn)] = v;
    }
    fft_dit(s, stw, lines, logn, true);
    for (int t = threadIdx.x; t < lines * nx; t += blockDim.x) {
        int l = t / nx, x = t - l * nx;
        long long row = row0 + l;
        if (row >= nrows) continue;
        phi[x + (long long)nx * row] = (double)s[l * N + x].x;
    }
}

// Host: the five passes of one solve.  smem_complex: complex elements of
// line storage per CTA; K: Khat (real, (nx+1)(ny+1)(nz+1)); t1..t3: twiddles
// of the doubled lengths; W1, W2: workspaces of (nx+1)ny nz and (nx+1)N2 nz.
inline int fft_ilog2(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

// dynamic shared memory limit of the four line kernels, once per device
template <class C>
bsn_status line_attrs(bsn_ctx* ctx, int smem_complex) {
    static bool attr[64] = {false};
    const int dev = ctx->device & 63;
    if (!attr[dev]) {
        int bytes = (int)(sizeof(C) * (smem_complex + 2048));
        const void* ks[] = {(const void*)fwd_x_kernel<C>, (const void*)axis_kernel<C>, (const void*)z_conv_kernel<C>,
                            (const void*)inv_x_kernel<C>};
        for (const void* k : ks)
            BSN_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        attr[dev] = true;
    }
    return BSN_OK;
}

template <class C>
bsn_status solve_lines(bsn_ctx* ctx, const RhoSrc& src, const typename Cx<C>::R* K, const C* t1, const C* t2,
                       const C* t3, C* W1, C* W2, double* phi, int smem_complex, int nt) {
    BSN_TRY(line_attrs<C>(ctx, smem_complex));
    const int nx = src.nx, ny = src.ny, nz = src.nz;
    const int N1 = 2 * nx, N2 = 2 * ny, N3 = 2 * nz;
    auto lines_for = [&](int N) { return std::max(1, std::min(64, smem_complex / N)); };
    auto smem_for = [&](int N, int lines) { return sizeof(C) * ((size_t)lines * N + N / 2); };
    int l1 = lines_for(N1), l2 = lines_for(N2), l3 = lines_for(N3);
    long long rows = (long long)ny * nz;
    prof_begin(ctx);
    fwd_x_kernel<C><<<grid1d(rows, l1), nt, smem_for(N1, l1), ctx->stream>>>(src, W1, t1, fft_ilog2(N1), l1);
    BSN_TRY(launch_check(ctx, "fwd_x_kernel"));
    int nbx2 = (nx + 1 + l2 - 1) / l2;
    AxisIO<C> y1{W1, W2, nx + 1, nz, nx + 1, nx + 1, (long long)(nx + 1) * ny, (long long)(nx + 1) * N2, ny, N2};
    prof_begin(ctx);
    axis_kernel<C><<<(unsigned)(nbx2 * nz), nt, smem_for(N2, l2), ctx->stream>>>(y1, t2, fft_ilog2(N2), l2, 0);
    BSN_TRY(launch_check(ctx, "fft_y_kernel"));
    int nbx3 = (nx + 1 + l3 - 1) / l3;
    prof_begin(ctx);
    z_conv_kernel<C><<<(unsigned)(nbx3 * N2), nt, smem_for(N3, l3), ctx->stream>>>(W2, K, nx, N2, ny, nz,
                                                                                    fft_ilog2(N3), l3, t3, 0, N2);
    BSN_TRY(launch_check(ctx, "z_conv_kernel"));
    AxisIO<C> y2{W2, W1, nx + 1, nz, nx + 1, nx + 1, (long long)(nx + 1) * N2, (long long)(nx + 1) * ny, N2, ny};
    prof_begin(ctx);
    axis_kernel<C><<<(unsigned)(nbx2 * nz), nt, smem_for(N2, l2), ctx->stream>>>(y2, t2, fft_ilog2(N2), l2, 1);
    BSN_TRY(launch_check(ctx, "fft_y_kernel"));
    prof_begin(ctx);
    inv_x_kernel<C><<<grid1d(rows, l1), nt, smem_for(N1, l1), ctx->stream>>>(W1, phi, nx, ny, nz, fft_ilog2(N1), l1,
                                                                              t1);
    return launch_check(ctx, "inv_x_kernel");
}

// The solve split at the z transform, for a z-slab decomposition (one rank
// per slab of nzl planes; the kernels and their per-line arithmetic are those
// of solve_lines, so the assembled potential is bit-identical to it).
// Forward: x and y transforms of the slab's nzl density planes into
// W2[kx + (nx+1)*(ky + N2*z)], z < nzl (W1: (nx+1) ny nzl scratch).
template <class C>
bsn_status slab_forward_lines(bsn_ctx* ctx, const RhoSrc& src, const C* t1, const C* t2, C* W1, C* W2,
                              int smem_complex, int nt) {
    BSN_TRY(line_attrs<C>(ctx, smem_complex));
    const int nx = src.nx, ny = src.ny, nz = src.nz;
    const int N1 = 2 * nx, N2 = 2 * ny;
    auto lines_for = [&](int N) { return std::max(1, std::min(64, smem_complex / N)); };
    auto smem_for = [&](int N, int lines) { return sizeof(C) * ((size_t)lines * N + N / 2); };
    int l1 = lines_for(N1), l2 = lines_for(N2);
    long long rows = (long long)ny * nz;
    prof_begin(ctx);
    fwd_x_kernel<C><<<grid1d(rows, l1), nt, smem_for(N1, l1), ctx->stream>>>(src, W1, t1, fft_ilog2(N1), l1);
    BSN_TRY(launch_check(ctx, "fwd_x_kernel"));
    int nbx2 = (nx + 1 + l2 - 1) / l2;
    AxisIO<C> y1{W1, W2, nx + 1, nz, nx + 1, nx + 1, (long long)(nx + 1) * ny, (long long)(nx + 1) * N2, ny, N2};
    prof_begin(ctx);
    axis_kernel<C><<<(unsigned)(nbx2 * nz), nt, smem_for(N2, l2), ctx->stream>>>(y1, t2, fft_ilog2(N2), l2, 0);
    return launch_check(ctx, "fft_y_kernel");
}

// z lines of the global grid (nz planes) for ky in [ky0, ky0 + nky), in place
// in T[kx + (nx+1)*(kyl + nky*z)].
template <class C>
bsn_status slab_zconv_lines(bsn_ctx* ctx, C* T, const typename Cx<C>::R* K, const C* t3, int nx, int ny, int nz,
                            int ky0, int nky, int smem_complex, int nt) {
    BSN_TRY(line_attrs<C>(ctx, smem_complex));
    const int N2 = 2 * ny, N3 = 2 * nz;
    auto lines_for = [&](int N) { return std::max(1, std::min(64, smem_complex / N)); };
    auto smem_for = [&](int N, int lines) { return sizeof(C) * ((size_t)lines * N + N / 2); };
    int l3 = lines_for(N3);
    int nbx3 = (nx + 1 + l3 - 1) / l3;
    if (nky < 1) return BSN_OK;
    prof_begin(ctx);
    z_conv_kernel<C><<<(unsigned)(nbx3 * nky), nt, smem_for(N3, l3), ctx->stream>>>(T, K, nx, N2, ny, nz,
                                                                                     fft_ilog2(N3), l3, t3, ky0, nky);
    return launch_check(ctx, "z_conv_kernel");
}

// Inverse: y and x transforms of the slab's W2 (z < nzl) into its nzl planes
// of Phi (W1: (nx+1) ny nzl scratch; W2 is left as it was).
template <class C>
bsn_status slab_inverse_lines(bsn_ctx* ctx, const C* W2, const C* t1, const C* t2, C* W1, double* phi, int nx,
                              int ny, int nz, int smem_complex, int nt) {
    BSN_TRY(line_attrs<C>(ctx, smem_complex));
    const int N1 = 2 * nx, N2 = 2 * ny;
    auto lines_for = [&](int N) { return std::max(1, std::min(64, smem_complex / N)); };
    auto smem_for = [&](int N, int lines) { return sizeof(C) * ((size_t)lines * N + N / 2); };
    int l1 = lines_for(N1), l2 = lines_for(N2);
    long long rows = (long long)ny * nz;
    int nbx2 = (nx + 1 + l2 - 1) / l2;
    AxisIO<C> y2{W2, W1, nx + 1, nz, nx + 1, nx + 1, (long long)(nx + 1) * N2, (long long)(nx + 1) * ny, N2, ny};
    prof_begin(ctx);
    axis_kernel<C><<<(unsigned)(nbx2 * nz), nt, smem_for(N2, l2), ctx->stream>>>(y2, t2, fft_ilog2(N2), l2, 1);
    BSN_TRY(launch_check(ctx, "fft_y_kernel"));
    prof_begin(ctx);
    inv_x_kernel<C><<<grid1d(rows, l1), nt, smem_for(N1, l1), ctx->stream>>>(W1, phi, nx, ny, nz, fft_ilog2(N1), l1,
                                                                              t1);
    return launch_check(ctx, "inv_x_kernel");
}

}  // namespace fft
}  // namespace bsn
