// sums.cuh -- the reductions of the driver's scalar results: compensated
// (double-double) grid sums, their block-parallel fixed-order merge, and the
// accrete! sums (src/sinks.jl:74-109) in the reference's sequential order.
#pragma once

#include "stage_f64.cuh"

namespace bsn {
namespace sums {

// two-sum compensated accumulator
struct DD { double hi, lo; };
__device__ __forceinline__ void dd_add(DD& s, double x) {
    double t = s.hi + x;
    double bp = t - s.hi;
    double e = (s.hi - (t - bp)) + (x - bp);
    s.hi = t;
    s.lo += e;
}
__device__ __forceinline__ DD dd_merge(DD a, DD b) {
    DD s = a;
    dd_add(s, b.hi);
    s.lo += b.lo;
    return s;
}

// Merge nblocks partial DD triples part[6 b + 2 d], part[6 b + 2 d + 1]
// (d = 0..2) with all NT threads of one block in a fixed order (thread t takes
// b = t, t + NT, ...; then a fixed shuffle tree and the warps in order), so
// the result does not depend on scheduling.  Thread 0 gets the merged pairs.
template <int NT>
__device__ void merge_partials3_pairs(const double* part, int nblocks, DD out[3]) {
    static_assert(NT % 32 == 0 && NT <= 1024, "block of whole warps");
    DD s[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    for (int b = threadIdx.x; b < nblocks; b += NT)
        for (int d = 0; d < 3; ++d) s[d] = dd_merge(s[d], DD{part[6 * b + 2 * d], part[6 * b + 2 * d + 1]});
    __shared__ DD red[3][NT / 32];
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o > 0; o >>= 1) {
            DD other = {__shfl_xor_sync(0xffffffffu, s[d].hi, o), __shfl_xor_sync(0xffffffffu, s[d].lo, o)};
            s[d] = dd_merge(s[d], other);
        }
        if ((threadIdx.x & 31) == 0) red[d][threadIdx.x >> 5] = s[d];
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) {
            DD acc = red[d][0];
            for (int w = 1; w < NT / 32; ++w) acc = dd_merge(acc, red[d][w]);
            out[d] = acc;
        }
}

// As merge_partials3_pairs; thread 0 gets out[d] = hi + lo.
template <int NT>
__device__ void merge_partials3(const double* part, int nblocks, double out[3]) {
    DD s[3];
    merge_partials3_pairs<NT>(part, nblocks, s);
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) out[d] = s[d].hi + s[d].lo;
}

// As merge_partials3_pairs; thread 0 gets out[2 d] = hi, out[2 d + 1] = lo.
template <int NT>
__device__ void merge_partials3_dd(const double* part, int nblocks, double out[6]) {
    DD s[3];
    merge_partials3_pairs<NT>(part, nblocks, s);
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) { out[2 * d] = s[d].hi; out[2 * d + 1] = s[d].lo; }
}

// accrete! sums over the active-index box [ilo,ihi] x [jlo,jhi] x [klo,khi]:
// cells with |x - p| < rs and rho > rho_min add rho * rate (and m * rate).
// The block evaluates the cells' terms in parallel, 1024 at a time, and
// thread 0 adds them in the reference's (k, j, i) order; a skipped cell adds
// +0.0, which leaves every sum as skipping it would (an accumulator that
// starts at +0.0 never becomes -0.0 by adding +0.0 or -0.0).  Thread 0 gets
// out = {dm, dPx, dPy, dPz}.
template <int NT>
__device__ void sink_sums(const double* U, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                          double y0, double z0, double px, double py, double pz, double rs, double rate,
                          double rho_min, int ilo, int ihi, int jlo, int jhi, int klo, int khi, double out[4]) {
    constexpr int CH = 1024;
    __shared__ double term[4][CH];
    const long long nI = ihi - ilo + 1, nJ = jhi - jlo + 1, nK = khi - klo + 1;
    const long long total = (nI > 0 && nJ > 0 && nK > 0) ? nI * nJ * nK : 0;
    Geom G(nx, ny, nz);
    double dm = 0.0, dPx = 0.0, dPy = 0.0, dPz = 0.0;
    for (long long base = 0; base < total; base += CH) {
        for (int e = threadIdx.x; e < CH; e += NT) {
            long long t = base + e;
            double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
            if (t < total) {
                int a = ilo + (int)(t % nI);
                long long rr = t / nI;
                int b = jlo + (int)(rr % nJ), c = klo + (int)(rr / nJ);
                double xc, yc, zc;
                f64::cell_xyz(a, b, c, x0, y0, z0, dx, dy, dz, xc, yc, zc);
                double r = sqrt(sq(xc - px) + sq(yc - py) + sq(zc - pz));
                if (!(r >= rs)) {
                    long long o = G.act(a, b, c);
                    if (!(U[o] <= rho_min)) {
                        v0 = U[o] * rate;
                        v1 = U[o + 1] * rate;
                        v2 = U[o + 2] * rate;
                        v3 = U[o + 3] * rate;
                    }
                }
            }
            term[0][e] = v0; term[1][e] = v1; term[2][e] = v2; term[3][e] = v3;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int m = (int)((total - base) < CH ? (total - base) : CH);
            for (int e = 0; e < m; ++e) {
                dm += term[0][e];
                dPx += term[1][e];
                dPy += term[2][e];
                dPz += term[3][e];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = dm; out[1] = dPx; out[2] = dPy; out[3] = dPz; }
}

}  // namespace sums
}  // namespace bsn
