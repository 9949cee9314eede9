// diagnostics.cu -- the driver's conserved-total and bound-mass diagnostics
// (src/diagnostics.jl) as one FP64 device reduction over the active cells:
// gas_energy_total, gas_kinetic_total, gas_momentum_total,
// gas_angular_momentum_total, bound_gas_mass and the gas mass.  Per-cell terms
// are the reference's expressions (built with -fmad=false); the whole-grid sums
// are compensated (two-sum), i.e. within about one rounding of the exact sum
// (the reference's own `sum` is pairwise, so no summation order is "the" one).
#include "diagnostics.cuh"
#include "sums.cuh"

namespace bsn {
namespace diag {

using sums::DD;
using sums::dd_add;
using sums::dd_merge;

__global__ void diag_kernel(const double* U, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                            double y0, double z0, const bsn_bh* bhs, const int* nbh_dev, int nbh, double g,
                            const int* done, double* part) {
    if (done && *done) return;
    const int nb = nbh_dev ? *nbh_dev : nbh;
    Geom G(nx, ny, nz);
    DD s[NDIAG];
#pragma unroll
    for (int q = 0; q < NDIAG; ++q) s[q] = DD{0.0, 0.0};
    long long n = (long long)nx * ny * nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int a = (int)(t % nx); long long rr = t / nx; int b = (int)(rr % ny); int c = (int)(rr / ny);
        long long o = G.act(a, b, c);
        double r = U[o], mx = U[o + 1], my = U[o + 2], mz = U[o + 3], E = U[o + 4];
        double xc, yc, zc;
        f64::cell_xyz(a, b, c, x0, y0, z0, dx, dy, dz, xc, yc, zc);
        double rs = jmax(r, 1e-30);
        double ke = 0.5 * (sq(mx) + sq(my) + sq(mz)) / rs;
        dd_add(s[0], E);
        dd_add(s[1], ke);
        dd_add(s[2], mx); dd_add(s[3], my); dd_add(s[4], mz);
        dd_add(s[5], yc * mz - zc * my);
        dd_add(s[6], zc * mx - xc * mz);
        dd_add(s[7], xc * my - yc * mx);
        double P = jmax((g - 1.0) * (E - rs * ke), 0.0);
        double eint = P / ((g - 1.0) * rs);
        double phi = 0.0;
        for (int i = 0; i < nb; ++i)
            phi -= bhs[i].mass / sqrt(sq(xc - bhs[i].pos[0]) + sq(yc - bhs[i].pos[1]) + sq(zc - bhs[i].pos[2]) +
                                      sq(bhs[i].eps));
        double etot = ke + eint + phi;
        if (etot <= 0.0) dd_add(s[8], rs);
        dd_add(s[9], r);
    }
    __shared__ DD red[NDIAG][32];
#pragma unroll
    for (int q = 0; q < NDIAG; ++q) {
        for (int o = 16; o > 0; o >>= 1) {
            DD other = {__shfl_xor_sync(0xffffffffu, s[q].hi, o), __shfl_xor_sync(0xffffffffu, s[q].lo, o)};
            s[q] = dd_merge(s[q], other);
        }
        if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = s[q];
    }
    __syncthreads();
    if (threadIdx.x < NDIAG) {
        const int q = threadIdx.x;
        DD acc = red[q][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) acc = dd_merge(acc, red[q][w]);
        part[2 * (NDIAG * blockIdx.x + q)] = acc.hi;
        part[2 * (NDIAG * blockIdx.x + q) + 1] = acc.lo;
    }
}

// totals times dV -> out[0..NDIAG); with the device loop's counters, the
// record {t, dt, totals} at index steps - 1 when it is below cap.
__global__ void diag_finish(const double* part, int nblocks, double dV, double* out, const double* t,
                            const double* dt, const int* steps, const int* done, int cap, const double* ledger) {
    if (done && *done) return;
    const int q = threadIdx.x;
    if (q >= NDIAG || blockIdx.x != 0) return;
    DD acc = {0.0, 0.0};
    for (int b = 0; b < nblocks; ++b) acc = dd_merge(acc, DD{part[2 * (NDIAG * b + q)], part[2 * (NDIAG * b + q) + 1]});
    double v = (acc.hi + acc.lo) * dV;
    if (!steps) { out[q] = v; return; }
    const int k = *steps - 1;
    if (k < 0 || k >= cap) return;
    double* rec = out + (long long)NREC * k;
    if (q == 0) { rec[0] = *t; rec[1] = *dt; }
    rec[2 + q] = v;
    if (q < f64::LEDT_COUNT) rec[2 + NDIAG + q] = ledger ? ledger[q] : 0.0;
}

bsn_status launch(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                  double y0, double z0, const bsn_bh* bhs_dev, const int* nbh_dev, int nbh, double gamma,
                  double* part, double* out, const double* t, const double* dt, const int* steps, const int* done,
                  int cap, const double* ledger) {
    prof_begin(ctx);
    diag_kernel<<<BLOCKS, 256, 0, ctx->stream>>>(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, bhs_dev, nbh_dev, nbh, gamma,
                                                 done, part);
    BSN_TRY(launch_check(ctx, "diag_kernel"));
    diag_finish<<<1, 32, 0, ctx->stream>>>(part, BLOCKS, dx * dy * dz, out, t, dt, steps, done, cap, ledger);
    return launch_check(ctx, "diag_finish");
}

}  // namespace diag
}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_diagnostics_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy,
                                          double dz, double x0, double y0, double z0, const bsn_bh* bhs, int nbh,
                                          double gamma, double out[10]) {
    if (!ctx) return BSN_ERR_ARG;
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || !out || (nbh > 0 && !bhs)) return set_err(ctx, BSN_ERR_ARG, "null argument");
    if (nbh < 0 || nbh > f64::MAXBH) return set_err(ctx, BSN_ERR_UNSUPPORTED, "at most %d black holes", f64::MAXBH);
    bsn_status st;
    const size_t npart = 2 * diag::NDIAG * diag::BLOCKS;
    double* part = (double*)slot(ctx, SLOT_DIAG, sizeof(double) * (npart + 16) + sizeof(bsn_bh) * f64::MAXBH, &st);
    BSN_TRY(st);
    double* dout = part + npart;                      // 10 totals
    bsn_bh* db = (bsn_bh*)(part + npart + 16);        // the BHs
    double* h = (double*)pinned(ctx, 128 + sizeof(bsn_bh) * f64::MAXBH, &st); BSN_TRY(st);
    if (nbh > 0) {
        memcpy(h + 16, bhs, sizeof(bsn_bh) * nbh);
        BSN_CUDA(ctx, cudaMemcpyAsync(db, h + 16, sizeof(bsn_bh) * nbh, cudaMemcpyHostToDevice, ctx->stream));
    }
    BSN_TRY(diag::launch(ctx, U, nx, ny, nz, dx, dy, dz, x0, y0, z0, db, nullptr, nbh, gamma, part, dout, nullptr,
                         nullptr, nullptr, nullptr, 0));
    BSN_CUDA(ctx, cudaMemcpyAsync(h, dout, sizeof(double) * diag::NDIAG, cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < diag::NDIAG; ++q) out[q] = h[q];
    return BSN_OK;
}
