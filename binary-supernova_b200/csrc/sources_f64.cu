// sources_f64.cu -- BH gravity, sinks, self-gravity gradient, gas->BH force,
// accretion, host FP64 orbits and the coupled-step driver (FP64 parity path).
#include <cmath>
#include <algorithm>
#include <cstring>

#include "hydro_f64.cuh"
#include "poisson.cuh"
#include "stage_launch.cuh"
#include "sums.cuh"

namespace bsn {
namespace f64 {


// add_bh_gravity_source! (src/gpu_kernels.jl:199-230)
// k0: global index of the grid's first active plane when it is a z-slab of a
// larger grid (0 otherwise); cell centres use the global index, so a slab's
// cells take the undivided grid's arithmetic.
__global__ void bh_gravity_kernel(double* dU, const double* U, int nx, int ny, int nz, double dx, double dy,
                                  double dz, double x0, double y0, double z0, BHSrc bh, int k0) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nx * ny * nz) return;
    int a = (int)(t % nx); long long r = t / nx; int b = (int)(r % ny); int c = (int)(r / ny);
    Geom G(nx, ny, nz);
    long long o = G.act(a, b, c);
    double xc, yc, zc;
    cell_xyz(a, b, c + k0, x0, y0, z0, dx, dy, dz, xc, yc, zc);
    double rho = U[o], vx = U[o + 1] / rho, vy = U[o + 2] / rho, vz = U[o + 3] / rho;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int n = 0; n < bh.n; ++n) {
        double ddx = xc - bh.px[n], ddy = yc - bh.py[n], ddz = zc - bh.pz[n];
        double r2 = sq(ddx) + sq(ddy) + sq(ddz) + sq(bh.eps[n]);
        double r3 = r2 * sqrt(r2);
        double fac = -bh.mass[n] / r3;
        ax += fac * ddx; ay += fac * ddy; az += fac * ddz;
    }
    dU[o + 1] += rho * ax;
    dU[o + 2] += rho * ay;
    dU[o + 3] += rho * az;
    dU[o + 4] += rho * (vx * ax + vy * ay + vz * az);
}

// rotating_frame_source! / relax_damping_source! (src/relax_ic.jl:59-176) as
// standalone passes over the active cells (the stage kernel applies the same
// per-cell functions in its epilogue)
__global__ void relax_src_kernel(double* dU, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                                 double x0, double y0, double z0, int rot, double omega, double inv_td, double t_damp) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nx * ny * nz) return;
    int a = (int)(t % nx); long long r = t / nx; int b = (int)(r % ny); int c = (int)(r / ny);
    Geom G(nx, ny, nz);
    long long o = G.act(a, b, c);
    double xc, yc, zc;
    cell_xyz(a, b, c, x0, y0, z0, dx, dy, dz, xc, yc, zc);
    double d[5] = {dU[o], dU[o + 1], dU[o + 2], dU[o + 3], dU[o + 4]};
    if (rot) rot_frame_src(d, U[o], U[o + 1], U[o + 2], xc, yc, omega);
    else damp_src(d, U[o], U[o + 1], U[o + 2], U[o + 3], xc, yc, inv_td, t_damp, omega);
    for (int q = 1; q < 5; ++q) dU[o + q] = d[q];
}

// add_sink_sources! (src/gpu_kernels.jl:238-284)
__global__ void sink_kernel(double* dU, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                            double x0, double y0, double z0, SinkSrc sk, int k0) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nx * ny * nz) return;
    int a = (int)(t % nx); long long r = t / nx; int b = (int)(r % ny); int c = (int)(r / ny);
    Geom G(nx, ny, nz);
    long long o = G.act(a, b, c);
    double xc, yc, zc;
    cell_xyz(a, b, c + k0, x0, y0, z0, dx, dy, dz, xc, yc, zc);
    double rho = U[o], mx = U[o + 1], my = U[o + 2], mz = U[o + 3], E = U[o + 4];
    if (!(rho > sk.rho_min)) return;
    for (int n = 0; n < sk.n; ++n) {
        double ddx = xc - sk.px[n], ddy = yc - sk.py[n], ddz = zc - sk.pz[n];
        double rr = sqrt(sq(ddx) + sq(ddy) + sq(ddz));
        if (rr < sk.rs[n]) {
            double ts = sk.ts[n];
            dU[o] -= rho / ts;
            if (sk.torque_free) {
                double rx = ddx / rr, ry = ddy / rr, rz = ddz / rr;
                double vx = mx / rho, vy = my / rho, vz = mz / rho;
                double vrx = vx - sk.vx[n], vry = vy - sk.vy[n], vrz = vz - sk.vz[n];
                double v_r = vrx * rx + vry * ry + vrz * rz;
                double e_int = E / rho - 0.5 * (sq(vx) + sq(vy) + sq(vz));
                dU[o + 1] -= rho * v_r * rx / ts;
                dU[o + 2] -= rho * v_r * ry / ts;
                dU[o + 3] -= rho * v_r * rz / ts;
                dU[o + 4] -= (0.5 * rho * sq(v_r) + rho * e_int) / ts;
            } else {
                dU[o + 1] -= mx / ts; dU[o + 2] -= my / ts; dU[o + 3] -= mz / ts; dU[o + 4] -= E / ts;
            }
        }
    }
}

// _sg_gradient_kernel! (src/gpu_kernels.jl:291-319).  Plo / Phi (may be
// null): the plane of Phi just below / above the grid, when the grid is a
// z-slab of a larger one; the slab's edge planes then take the central
// difference the larger grid's cells take there.
__global__ void sg_gradient_kernel(double* dU, const double* U, const double* P, int nx, int ny, int nz,
                                   double i2x, double i2y, double i2z, const double* Plo = nullptr,
                                   const double* Phi = nullptr) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nx * ny * nz) return;
    int a = (int)(t % nx); long long r = t / nx; int b = (int)(r % ny); int c = (int)(r / ny);
    Geom G(nx, ny, nz);
    long long o = G.act(a, b, c);
    double rho = U[o], rvx = U[o + 1], rvy = U[o + 2], rvz = U[o + 3];
    int ip = min(a + 1, nx - 1), im = max(a - 1, 0);
    int jp = min(b + 1, ny - 1), jm = max(b - 1, 0);
    int kp = min(c + 1, nz - 1), km = max(c - 1, 0);
    double fx = ip > im ? i2x : 2.0 * i2x, fy = jp > jm ? i2y : 2.0 * i2y, fz = kp > km ? i2z : 2.0 * i2z;
    long long sy = nx, sz = (long long)nx * ny;
    double gx = (P[ip + sy * b + sz * c] - P[im + sy * b + sz * c]) * fx;
    double gy = (P[a + sy * jp + sz * c] - P[a + sy * jm + sz * c]) * fy;
    double pzp = P[a + sy * b + sz * kp], pzm = P[a + sy * b + sz * km];
    // with a neighbour plane the slab is part of a grid of >= 2 planes, where
    // every plane's z difference spans two distinct planes
    if (Plo || Phi) fz = i2z;
    if (c == nz - 1 && Phi) pzp = Phi[a + sy * b];
    if (c == 0 && Plo) pzm = Plo[a + sy * b];
    double gz = (pzp - pzm) * fz;
    double vdotg = (rvx * gx + rvy * gy + rvz * gz) / rho;
    dU[o + 1] -= rho * gx;
    dU[o + 2] -= rho * gy;
    dU[o + 3] -= rho * gz;
    dU[o + 4] -= rho * vdotg;
}

// Compensated (two-sum) accumulation: the parallel sum is accurate to about
// one rounding of the exact sum, i.e. within the reference's own sequential
// rounding error.
using sums::DD;
using sums::dd_add;
using sums::dd_merge;

// gas_force_on_bh (src/gravity_bh.jl:91-113): out[3*blocks] partial (hi,lo).
__global__ void gas_force_kernel(const double* U, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                                 double y0, double z0, double px, double py, double pz, double mass, double eps,
                                 double* part, int k0) {
    Geom G(nx, ny, nz);
    double dV = dx * dy * dz;
    DD s[3] = {{0, 0}, {0, 0}, {0, 0}};
    long long n = (long long)nx * ny * nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        int a = (int)(t % nx); long long r = t / nx; int b = (int)(r % ny); int c = (int)(r / ny);
        double xc, yc, zc;
        cell_xyz(a, b, c + k0, x0, y0, z0, dx, dy, dz, xc, yc, zc);
        double ddx = xc - px, ddy = yc - py, ddz = zc - pz;
        double r2 = sq(ddx) + sq(ddy) + sq(ddz) + sq(eps);
        double r3 = r2 * sqrt(r2);
        double fac = mass / r3 * U[G.act(a, b, c)] * dV;
        dd_add(s[0], fac * ddx);
        dd_add(s[1], fac * ddy);
        dd_add(s[2], fac * ddz);
    }
    __shared__ DD red[3][32];
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o > 0; o >>= 1) {
            DD other = {__shfl_xor_sync(0xffffffffu, s[d].hi, o), __shfl_xor_sync(0xffffffffu, s[d].lo, o)};
            s[d] = dd_merge(s[d], other);
        }
        if ((threadIdx.x & 31) == 0) red[d][threadIdx.x >> 5] = s[d];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int d = 0; d < 3; ++d) {
            DD acc = red[d][0];
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) acc = dd_merge(acc, red[d][w]);
            part[6 * blockIdx.x + 2 * d] = acc.hi;
            part[6 * blockIdx.x + 2 * d + 1] = acc.lo;
        }
    }
}

__global__ void gas_force_finish(const double* part, int nblocks, double* out, int as_pairs) {
    if (as_pairs) {   // the compensated (hi, lo) pairs of the grid, for a merge over slabs
        double F[6];
        sums::merge_partials3_dd<256>(part, nblocks, F);
        if (threadIdx.x == 0)
            for (int d = 0; d < 6; ++d) out[d] = F[d];
        return;
    }
    double F[3];
    sums::merge_partials3<256>(part, nblocks, F);
    if (threadIdx.x == 0) { out[0] = F[0]; out[1] = F[1]; out[2] = F[2]; }
}

// accrete!'s per-cell terms (src/sinks.jl:74-109) over the global active box
// [ilo,ihi] x [jlo,jhi] x [klo,khi] restricted to this grid's planes (global
// k0 .. k0 + nz - 1), in the reference's (k, j, i) order: {rho, mx, my, mz} *
// rate inside the sink sphere where rho > rho_min, zeros elsewhere (adding
// +0.0 leaves the sequential sums as skipping the cell does).
__global__ void sink_terms_kernel(const double* U, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                                  double y0, double z0, int k0, double px, double py, double pz, double rs,
                                  double rate, double rho_min, int ilo, int ihi, int jlo, int jhi, int klo, int khi,
                                  double* out) {
    const long long nI = ihi - ilo + 1, nJ = jhi - jlo + 1, nK = khi - klo + 1;
    const long long total = nI * nJ * nK;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int a = ilo + (int)(t % nI);
    long long rr = t / nI;
    int b = jlo + (int)(rr % nJ), kg = klo + (int)(rr / nJ);
    double xc, yc, zc;
    cell_xyz(a, b, kg, x0, y0, z0, dx, dy, dz, xc, yc, zc);
    double r = sqrt(sq(xc - px) + sq(yc - py) + sq(zc - pz));
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (!(r >= rs)) {
        long long o = Geom(nx, ny, nz).act(a, b, kg - k0);
        if (!(U[o] <= rho_min))
            for (int q = 0; q < 4; ++q) v[q] = U[o + q] * rate;
    }
    for (int q = 0; q < 4; ++q) out[4 * t + q] = v[q];
}

// accrete! sums (src/sinks.jl:74-109) in the reference's exact loop order
// over the (k,j,i) bounding box of the sink sphere (sums::sink_sums), so the
// sequential sum is reproduced bit for bit.
__global__ void accrete_kernel(const double* U, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                               double y0, double z0, double px, double py, double pz, double rs, double rate,
                               double rho_min, int ilo, int ihi, int jlo, int jhi, int klo, int khi, double* out) {
    double v[4];
    sums::sink_sums<256>(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, px, py, pz, rs, rate, rho_min, ilo, ihi, jlo, jhi,
                         klo, khi, v);
    if (threadIdx.x == 0) { out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; out[3] = v[3]; }
}

}  // namespace f64

using namespace f64;

static bsn_status fill_bh(bsn_ctx* ctx, const bsn_bh* bhs, int nbh, BHSrc& s) {
    if (nbh < 0 || nbh > MAXBH) return set_err(ctx, BSN_ERR_UNSUPPORTED, "at most %d black holes (got %d)", MAXBH, nbh);
    if (nbh > 0 && !bhs) return set_err(ctx, BSN_ERR_ARG, "bhs is null");
    memset(&s, 0, sizeof(s));
    s.n = nbh;
    for (int n = 0; n < nbh; ++n) {
        s.px[n] = bhs[n].pos[0]; s.py[n] = bhs[n].pos[1]; s.pz[n] = bhs[n].pos[2];
        s.mass[n] = bhs[n].mass; s.eps[n] = bhs[n].eps;
    }
    return BSN_OK;
}

static bsn_status fill_sink(bsn_ctx* ctx, const bsn_bh* bhs, int nbh, double f_sink, int torque_free,
                            double rho_min, SinkSrc& s) {
    if (nbh < 0 || nbh > MAXBH) return set_err(ctx, BSN_ERR_UNSUPPORTED, "at most %d black holes (got %d)", MAXBH, nbh);
    if (nbh > 0 && !bhs) return set_err(ctx, BSN_ERR_ARG, "bhs is null");
    memset(&s, 0, sizeof(s));
    s.n = nbh; s.torque_free = torque_free ? 1 : 0; s.rho_min = rho_min;
    for (int n = 0; n < nbh; ++n) {
        s.px[n] = bhs[n].pos[0]; s.py[n] = bhs[n].pos[1]; s.pz[n] = bhs[n].pos[2];
        s.vx[n] = bhs[n].vel[0]; s.vy[n] = bhs[n].vel[1]; s.vz[n] = bhs[n].vel[2];
        s.rs[n] = bh_r_sink(bhs[n]); s.ts[n] = bh_t_sink(bhs[n], f_sink);
    }
    return BSN_OK;
}

// out[3] = the force, or with pairs != 0 out[6] = its compensated (hi, lo)
// pairs per component; k0 as bh_gravity_kernel's.
static bsn_status gas_force(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                            const bsn_bh& bh, double x0, double y0, double z0, double* out, int k0 = 0,
                            int pairs = 0) {
    const int blocks = 148 * 4;
    bsn_status st;
    double* part = (double*)slot(ctx, SLOT_RED, sizeof(double) * (6 * blocks + 8), &st); BSN_TRY(st);
    gas_force_kernel<<<blocks, 256, 0, ctx->stream>>>(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, bh.pos[0], bh.pos[1],
                                                      bh.pos[2], bh.mass, bh.eps, part, k0);
    BSN_TRY(launch_check(ctx, "gas_force_kernel"));
    gas_force_finish<<<1, 256, 0, ctx->stream>>>(part, blocks, part + 6 * blocks, pairs);
    BSN_TRY(launch_check(ctx, "gas_force_finish"));
    double* h = (double*)pinned(ctx, 64, &st); BSN_TRY(st);
    const int nout = pairs ? 6 : 3;
    BSN_CUDA(ctx, cudaMemcpyAsync(h, part + 6 * blocks, 8 * nout, cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int d = 0; d < nout; ++d) out[d] = h[d];
    return BSN_OK;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Conservative active-index box [b0,b1] x [b2,b3] x [b4,b5] (0-based,
// inclusive) of the sink sphere |x - p| < r_sink on an nx x ny x nz grid; the
// whole grid for a non-finite sink geometry (the reference then selects no
// cell by r >= rs, which is false for NaN, so every cell's NaN enters its sums).
static void sink_box(const bsn_bh& bh, double rs, int nx, int ny, int nz, double dx, double dy, double dz, double x0,
                     double y0, double z0, int b[6]) {
    auto lo = [](double p, double r, double o, double h) { return (int)std::floor((p - r - o) / h) - 2; };
    auto hi = [](double p, double r, double o, double h) { return (int)std::ceil((p + r - o) / h) + 2; };
    b[0] = clampi(lo(bh.pos[0], rs, x0, dx), 0, nx - 1); b[1] = clampi(hi(bh.pos[0], rs, x0, dx), 0, nx - 1);
    b[2] = clampi(lo(bh.pos[1], rs, y0, dy), 0, ny - 1); b[3] = clampi(hi(bh.pos[1], rs, y0, dy), 0, ny - 1);
    b[4] = clampi(lo(bh.pos[2], rs, z0, dz), 0, nz - 1); b[5] = clampi(hi(bh.pos[2], rs, z0, dz), 0, nz - 1);
    if (!std::isfinite(rs) || !std::isfinite(bh.pos[0]) || !std::isfinite(bh.pos[1]) || !std::isfinite(bh.pos[2])) {
        b[0] = 0; b[1] = nx - 1; b[2] = 0; b[3] = ny - 1; b[4] = 0; b[5] = nz - 1;
    }
}

// The end of accrete! (src/sinks.jl:96-107) from its sums.
static void accrete_update(bsn_bh* bh, double dm, double dPx, double dPy, double dPz) {
    if (dm > 0.0) {
        double M_new = bh->mass + dm;
        bh->vel[0] = (bh->mass * bh->vel[0] + dPx) / M_new;
        bh->vel[1] = (bh->mass * bh->vel[1] + dPy) / M_new;
        bh->vel[2] = (bh->mass * bh->vel[2] + dPz) / M_new;
        bh->mass = M_new;
    }
}

static bsn_status accrete(bsn_ctx* ctx, bsn_bh* bh, const double* U, int nx, int ny, int nz, double dx, double dy,
                          double dz, double x0, double y0, double z0, double dt, double f_sink, double rho_min) {
    double rs = bh_r_sink(*bh), ts = bh_t_sink(*bh, f_sink);
    double dV = dx * dy * dz;
    double rate = dV / ts * dt;
    int b[6];
    sink_box(*bh, rs, nx, ny, nz, dx, dy, dz, x0, y0, z0, b);
    const int ilo = b[0], ihi = b[1], jlo = b[2], jhi = b[3], klo = b[4], khi = b[5];
    bsn_status st;
    double* d = (double*)slot(ctx, SLOT_RED, 64, &st); BSN_TRY(st);
    accrete_kernel<<<1, 256, 0, ctx->stream>>>(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, bh->pos[0], bh->pos[1],
                                              bh->pos[2], rs, rate, rho_min, ilo, ihi, jlo, jhi, klo, khi, d);
    BSN_TRY(launch_check(ctx, "accrete_kernel"));
    double* h = (double*)pinned(ctx, 64, &st); BSN_TRY(st);
    BSN_CUDA(ctx, cudaMemcpyAsync(h, d, 32, cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    accrete_update(bh, h[0], h[1], h[2], h[3]);
    return BSN_OK;
}

// ---- host FP64 orbits -------------------------------------------------------
// src/nbody.jl:24-56
static void nbody_rhs(double (*dp)[3], double (*dv)[3], const bsn_bh* b, int n, const double* Fg) {
    for (int i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) dp[i][d] = b[i].vel[d];
        double a[3] = {Fg[3 * i] / b[i].mass, Fg[3 * i + 1] / b[i].mass, Fg[3 * i + 2] / b[i].mass};
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            double x = b[j].pos[0] - b[i].pos[0], y = b[j].pos[1] - b[i].pos[1], z = b[j].pos[2] - b[i].pos[2];
            double r2 = x * x + y * y + z * z + b[j].eps * b[j].eps;
            double r3 = r2 * std::sqrt(r2);
            double fac = b[j].mass / r3;
            a[0] = a[0] + fac * x; a[1] = a[1] + fac * y; a[2] = a[2] + fac * z;
        }
        for (int d = 0; d < 3; ++d) dv[i][d] = a[d];
    }
}

}  // namespace bsn

using namespace bsn;

extern "C" bsn_status bsn_add_bh_gravity_source_f64(bsn_ctx* ctx, double* dU, const double* U, int nx, int ny, int nz,
                                                    double dx, double dy, double dz, const bsn_bh* bhs, int nbh,
                                                    double x0, double y0, double z0) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!dU || !U) return set_err(ctx, BSN_ERR_ARG, "null array");
    BHSrc s;
    BSN_TRY(fill_bh(ctx, bhs, nbh, s));
    bh_gravity_kernel<<<grid1d((long long)nx * ny * nz, 256), 256, 0, ctx->stream>>>(dU, U, nx, ny, nz, dx, dy, dz,
                                                                                       x0, y0, z0, s, 0);
    return launch_check(ctx, "bh_gravity_kernel");
}

extern "C" bsn_status bsn_rotating_frame_source_f64(bsn_ctx* ctx, double* dU, const double* U, int nx, int ny,
                                                    int nz, double dx, double dy, double dz, double x0, double y0,
                                                    double z0, double Omega) {
    if (!ctx) return BSN_ERR_ARG;
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!dU || !U) return set_err(ctx, BSN_ERR_ARG, "null array");
    relax_src_kernel<<<grid1d((long long)nx * ny * nz, 256), 256, 0, ctx->stream>>>(dU, U, nx, ny, nz, dx, dy, dz, x0,
                                                                                      y0, z0, 1, Omega, 0.0, 0.0);
    return launch_check(ctx, "relax_src_kernel");
}

extern "C" bsn_status bsn_relax_damping_source_f64(bsn_ctx* ctx, double* dU, const double* U, int nx, int ny, int nz,
                                                   double dx, double dy, double dz, double x0, double y0, double z0,
                                                   double t_damp, double Omega) {
    if (!ctx) return BSN_ERR_ARG;
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!dU || !U) return set_err(ctx, BSN_ERR_ARG, "null array");
    if (!(t_damp > 0.0)) return set_err(ctx, BSN_ERR_ARG, "t_damp must be positive");
    relax_src_kernel<<<grid1d((long long)nx * ny * nz, 256), 256, 0, ctx->stream>>>(dU, U, nx, ny, nz, dx, dy, dz, x0,
                                                                                      y0, z0, 0, Omega, 1.0 / t_damp,
                                                                                      t_damp);
    return launch_check(ctx, "relax_src_kernel");
}

extern "C" bsn_status bsn_add_sink_sources_f64(bsn_ctx* ctx, double* dU, const double* U, int nx, int ny, int nz,
                                               double dx, double dy, double dz, const bsn_bh* bhs, int nbh, double x0,
                                               double y0, double z0, double f_sink, int torque_free,
                                               double rho_sink_min) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!dU || !U) return set_err(ctx, BSN_ERR_ARG, "null array");
    SinkSrc s;
    BSN_TRY(fill_sink(ctx, bhs, nbh, f_sink, torque_free, rho_sink_min, s));
    sink_kernel<<<grid1d((long long)nx * ny * nz, 256), 256, 0, ctx->stream>>>(dU, U, nx, ny, nz, dx, dy, dz, x0, y0,
                                                                                 z0, s, 0);
    return launch_check(ctx, "sink_kernel");
}

extern "C" bsn_status bsn_gas_force_on_bh_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx,
                                              double dy, double dz, const bsn_bh* bh, double x0, double y0, double z0,
                                              double out[3]) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || !bh || !out) return set_err(ctx, BSN_ERR_ARG, "null argument");
    return gas_force(ctx, U, nx, ny, nz, dx, dy, dz, *bh, x0, y0, z0, out);
}

extern "C" bsn_status bsn_accrete_f64(bsn_ctx* ctx, bsn_bh* bh, const double* U, int nx, int ny, int nz, double dx,
                                      double dy, double dz, double x0, double y0, double z0, double dt, double f_sink,
                                      double rho_sink_min) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || !bh) return set_err(ctx, BSN_ERR_ARG, "null argument");
    return accrete(ctx, bh, U, nx, ny, nz, dx, dy, dz, x0, y0, z0, dt, f_sink, rho_sink_min);
}

// ---- the sources on a z-slab of a larger grid (k0: its first global plane) ----

extern "C" bsn_status bsn_add_bh_gravity_source_slab_f64(bsn_ctx* ctx, double* dU, const double* U, int nx, int ny,
                                                         int nz, double dx, double dy, double dz, const bsn_bh* bhs,
                                                         int nbh, double x0, double y0, double z0, int k0) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!dU || !U) return set_err(ctx, BSN_ERR_ARG, "null array");
    if (k0 < 0) return set_err(ctx, BSN_ERR_ARG, "k0 = %d", k0);
    BHSrc s;
    BSN_TRY(fill_bh(ctx, bhs, nbh, s));
    bh_gravity_kernel<<<grid1d((long long)nx * ny * nz, 256), 256, 0, ctx->stream>>>(dU, U, nx, ny, nz, dx, dy, dz,
                                                                                       x0, y0, z0, s, k0);
    return launch_check(ctx, "bh_gravity_kernel");
}

extern "C" bsn_status bsn_add_sink_sources_slab_f64(bsn_ctx* ctx, double* dU, const double* U, int nx, int ny, int nz,
                                                    double dx, double dy, double dz, const bsn_bh* bhs, int nbh,
                                                    double x0, double y0, double z0, double f_sink, int torque_free,
                                                    double rho_sink_min, int k0) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!dU || !U) return set_err(ctx, BSN_ERR_ARG, "null array");
    if (k0 < 0) return set_err(ctx, BSN_ERR_ARG, "k0 = %d", k0);
    SinkSrc s;
    BSN_TRY(fill_sink(ctx, bhs, nbh, f_sink, torque_free, rho_sink_min, s));
    sink_kernel<<<grid1d((long long)nx * ny * nz, 256), 256, 0, ctx->stream>>>(dU, U, nx, ny, nz, dx, dy, dz, x0, y0,
                                                                                 z0, s, k0);
    return launch_check(ctx, "sink_kernel");
}

extern "C" bsn_status bsn_gas_force_on_bh_slab_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx,
                                                   double dy, double dz, const bsn_bh* bh, double x0, double y0,
                                                   double z0, int k0, double out[6]) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || !bh || !out) return set_err(ctx, BSN_ERR_ARG, "null argument");
    if (k0 < 0) return set_err(ctx, BSN_ERR_ARG, "k0 = %d", k0);
    return gas_force(ctx, U, nx, ny, nz, dx, dy, dz, *bh, x0, y0, z0, out, k0, 1);
}

extern "C" bsn_status bsn_merge_force_pairs(const double* pairs, int nparts, double out[3]) {
    if (!pairs || !out || nparts < 0) return BSN_ERR_ARG;
    for (int d = 0; d < 3; ++d) {
        // the two-sum merge of the device reduction (sums.cuh dd_merge), in part order
        double hi = 0.0, lo = 0.0;
        for (int p = 0; p < nparts; ++p) {
            const double x = pairs[6 * p + 2 * d], t = hi + x, bp = t - hi;
            lo += (hi - (t - bp)) + (x - bp);
            hi = t;
            lo += pairs[6 * p + 2 * d + 1];
        }
        out[d] = hi + lo;
    }
    return BSN_OK;
}

extern "C" bsn_status bsn_sink_box(const bsn_bh* bh, int nx, int ny, int nz, double dx, double dy, double dz,
                                   double x0, double y0, double z0, int box[6]) {
    if (!bh || !box || nx < 1 || ny < 1 || nz < 1) return BSN_ERR_ARG;
    sink_box(*bh, bh_r_sink(*bh), nx, ny, nz, dx, dy, dz, x0, y0, z0, box);
    return BSN_OK;
}

extern "C" bsn_status bsn_sink_terms_slab_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx,
                                              double dy, double dz, double x0, double y0, double z0, int k0,
                                              const bsn_bh* bh, double dt, double f_sink, double rho_sink_min,
                                              const int box[6], double* terms, long long cap, long long* count) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || !bh || !box || !count || (cap > 0 && !terms)) return set_err(ctx, BSN_ERR_ARG, "null argument");
    if (k0 < 0) return set_err(ctx, BSN_ERR_ARG, "k0 = %d", k0);
    const int klo = std::max(box[4], k0), khi = std::min(box[5], k0 + nz - 1);
    if (box[0] < 0 || box[1] >= nx || box[2] < 0 || box[3] >= ny)
        return set_err(ctx, BSN_ERR_ARG, "sink box outside the grid's x/y range");
    const long long n = (box[1] >= box[0] && box[3] >= box[2] && khi >= klo)
                            ? (long long)(box[1] - box[0] + 1) * (box[3] - box[2] + 1) * (khi - klo + 1) : 0;
    *count = n;
    if (n == 0) return BSN_OK;
    if (n > cap) return set_err(ctx, BSN_ERR_ARG, "%lld sink cells, room for %lld", n, cap);
    const double rs = bh_r_sink(*bh), ts = bh_t_sink(*bh, f_sink);
    const double rate = dx * dy * dz / ts * dt;
    bsn_status st;
    double* d = (double*)slot(ctx, SLOT_RED, sizeof(double) * 4 * (size_t)n, &st); BSN_TRY(st);
    sink_terms_kernel<<<grid1d(n, 256), 256, 0, ctx->stream>>>(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, k0,
                                                                bh->pos[0], bh->pos[1], bh->pos[2], rs, rate,
                                                                rho_sink_min, box[0], box[1], box[2], box[3], klo,
                                                                khi, d);
    BSN_TRY(launch_check(ctx, "sink_terms_kernel"));
    BSN_CUDA(ctx, cudaMemcpyAsync(terms, d, sizeof(double) * 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    BSN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BSN_OK;
}

extern "C" bsn_status bsn_accrete_from_terms(bsn_bh* bh, const double* terms, long long n) {
    if (!bh || (n > 0 && !terms) || n < 0) return BSN_ERR_ARG;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long c = 0; c < n; ++c)
        for (int q = 0; q < 4; ++q) s[q] += terms[4 * c + q];
    accrete_update(bh, s[0], s[1], s[2], s[3]);
    return BSN_OK;
}

extern "C" bsn_status bsn_euler3d_stage(bsn_ctx* ctx, double* Uout, double* Uin, const double* Un, int nx, int ny,
                                        int nz, double dx, double dy, double dz, double dt, double gamma, int stage,
                                        double rho_floor, double P_floor, int precision,
                                        const bsn_stage_sources* src) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!Uout || !Uin || !Un) return set_err(ctx, BSN_ERR_ARG, "null state array");
    if (Uout == Uin) return set_err(ctx, BSN_ERR_ARG, "Uout must not be the stage input (the stencils read it)");
    if (stage < 1 || stage > 3) return set_err(ctx, BSN_ERR_ARG, "stage %d outside 1..3", stage);
    if (precision != PREC_F64 && precision != PREC_F32 && precision != PREC_LEARNED)
        return set_err(ctx, BSN_ERR_ARG, "unknown precision %d", precision);
    f64::StageArgs A;
    stage_args_init(A, nx, ny, nz, dx, dy, dz, gamma, BSN_BC_OUTFLOW, rho_floor, P_floor);
    A.Uin = Uin;
    A.Gh = Uin;   // the caller filled (and exchanged) the input's ghost cells
    A.Un = Un;
    A.Uout = Uout;
    A.mode = 0;
    set_stage(A, stage, dt);
    A.stiff_guard = ctx->stiff_guard;
    if (src) {
        if (src->k0 < 0) return set_err(ctx, BSN_ERR_ARG, "k0 = %d", src->k0);
        if (src->nsink < 0 || src->nsink > src->nbh) return set_err(ctx, BSN_ERR_ARG, "nsink %d of %d BHs", src->nsink, src->nbh);
        A.x0 = src->x0; A.y0 = src->y0; A.z0 = src->z0;
        A.k0 = src->k0;
        if (src->nbh > 0) {
            BSN_TRY(fill_bh(ctx, src->bhs, src->nbh, A.bh));
            A.use_bh = 1;
        }
        if (src->nsink > 0) {
            BSN_TRY(fill_sink(ctx, src->bhs, src->nsink, src->f_sink, src->torque_free, src->rho_sink_min, A.sk));
            A.use_sink = 1;
            A.stiff_guard = 1;   // near-vacuum cells beside the sinks (FP32 stencils)
        }
        if (src->phi) {
            A.phi = src->phi;
            A.use_sg = 1;
            A.phi_lo = src->phi_lo;
            A.phi_hi = src->phi_hi;
        }
    }
    BSN_TRY(stage_launch(ctx, precision, A));
    // the reference combines whole arrays: after stage 3 the ghost cells of U
    // hold (1/3) U^n's + (2/3) the stage input's (whose right-hand side is zero there)
    if (stage == 3 && Uout == Un) BSN_TRY(f64_ghost_combine(ctx, Uout, Uin, Uin, nx, ny, nz, BSN_BC_OUTFLOW, dt));
    return BSN_OK;
}

extern "C" bsn_status bsn_sg_gradient_f64(bsn_ctx* ctx, double* dU, const double* U, const double* phi, int nx, int ny,
                                          int nz, double dx, double dy, double dz) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!dU || !U || !phi) return set_err(ctx, BSN_ERR_ARG, "null array");
    sg_gradient_kernel<<<grid1d((long long)nx * ny * nz, 256), 256, 0, ctx->stream>>>(dU, U, phi, nx, ny, nz, 0.5 / dx,
                                                                                        0.5 / dy, 0.5 / dz);
    return launch_check(ctx, "sg_gradient_kernel");
}

extern "C" bsn_status bsn_sg_gradient_slab_f64(bsn_ctx* ctx, double* dU, const double* U, const double* phi,
                                               const double* phi_lo, const double* phi_hi, int nx, int ny, int nz,
                                               double dx, double dy, double dz) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!dU || !U || !phi) return set_err(ctx, BSN_ERR_ARG, "null array");
    sg_gradient_kernel<<<grid1d((long long)nx * ny * nz, 256), 256, 0, ctx->stream>>>(
        dU, U, phi, nx, ny, nz, 0.5 / dx, 0.5 / dy, 0.5 / dz, phi_lo, phi_hi);
    return launch_check(ctx, "sg_gradient_kernel");
}

extern "C" bsn_status bsn_add_self_gravity_source_f64(bsn_ctx* ctx, double* dU, const double* U, int nx, int ny,
                                                      int nz, double dx, double dy, double dz) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!dU || !U) return set_err(ctx, BSN_ERR_ARG, "null array");
    bsn_status st;
    double* phi = (double*)slot(ctx, SLOT_PHI, sizeof(double) * (size_t)nx * ny * nz, &st); BSN_TRY(st);
    BSN_TRY(poisson_from_state(ctx, U, nx, ny, nz, dx, dy, dz, -1.0, phi));
    return bsn_sg_gradient_f64(ctx, dU, U, phi, nx, ny, nz, dx, dy, dz);
}

extern "C" bsn_status bsn_nbody_step(bsn_bh* b, int n, double dt, const double* Fg) {
    if (!b || n < 1 || !Fg) return BSN_ERR_ARG;
    std::vector<double> p0(3 * n), v0(3 * n), p1(3 * n), v1(3 * n), p2(3 * n), v2(3 * n), dp(3 * n), dv(3 * n);
    auto DP = reinterpret_cast<double (*)[3]>(dp.data());
    auto DV = reinterpret_cast<double (*)[3]>(dv.data());
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) { p0[3 * i + d] = b[i].pos[d]; v0[3 * i + d] = b[i].vel[d]; }
    nbody_rhs(DP, DV, b, n, Fg);   // stage 1
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            p1[3 * i + d] = p0[3 * i + d] + dt * DP[i][d];
            v1[3 * i + d] = v0[3 * i + d] + dt * DV[i][d];
            b[i].pos[d] = p1[3 * i + d]; b[i].vel[d] = v1[3 * i + d];
        }
    nbody_rhs(DP, DV, b, n, Fg);   // stage 2
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            p2[3 * i + d] = 0.75 * p0[3 * i + d] + 0.25 * (p1[3 * i + d] + dt * DP[i][d]);
            v2[3 * i + d] = 0.75 * v0[3 * i + d] + 0.25 * (v1[3 * i + d] + dt * DV[i][d]);
        }
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) { b[i].pos[d] = p2[3 * i + d]; b[i].vel[d] = v2[3 * i + d]; }
    nbody_rhs(DP, DV, b, n, Fg);   // stage 3
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            b[i].pos[d] = (1.0 / 3.0) * p0[3 * i + d] + (2.0 / 3.0) * (p2[3 * i + d] + dt * DP[i][d]);
            b[i].vel[d] = (1.0 / 3.0) * v0[3 * i + d] + (2.0 / 3.0) * (v2[3 * i + d] + dt * DV[i][d]);
        }
    return BSN_OK;
}

extern "C" bsn_status bsn_kepler_init(const bsn_bh* b, const double com[3], const double* nhat, double Omega,
                                      double st[13]) {
    if (!b || !com || !st) return BSN_ERR_ARG;
    double dx = b[0].pos[0] - b[1].pos[0], dy = b[0].pos[1] - b[1].pos[1], dz = b[0].pos[2] - b[1].pos[2];
    if (!(std::sqrt(dx * dx + dy * dy + dz * dz) > 0)) return BSN_ERR_ARG;   // coincident BHs
    double rx = b[0].pos[0] - com[0], ry = b[0].pos[1] - com[1], rz = b[0].pos[2] - com[2];
    double vx = b[0].vel[0], vy = b[0].vel[1], vz = b[0].vel[2];
    double nh[3];
    if (!nhat) {
        double Lx = ry * vz - rz * vy, Ly = rz * vx - rx * vz, Lz = rx * vy - ry * vx;
        double Lm = std::sqrt(Lx * Lx + Ly * Ly + Lz * Lz);
        if (!(Lm > 0)) return BSN_ERR_ARG;   // zero angular momentum: nhat must be given
        nh[0] = Lx / Lm; nh[1] = Ly / Lm; nh[2] = Lz / Lm;
    } else {
        double nm = std::sqrt(nhat[0] * nhat[0] + nhat[1] * nhat[1] + nhat[2] * nhat[2]);
        if (!(std::fabs(nm - 1.0) < 1e-10)) return BSN_ERR_ARG;
        nh[0] = nhat[0]; nh[1] = nhat[1]; nh[2] = nhat[2];
    }
    double W = Omega;
    if (!(Omega > 0)) {
        double R = std::sqrt(rx * rx + ry * ry + rz * rz), V = std::sqrt(vx * vx + vy * vy + vz * vz);
        if (!(R > 0) || !(V > 0)) return BSN_ERR_ARG;
        W = V / R;
    }
    st[0] = com[0]; st[1] = com[1]; st[2] = com[2]; st[3] = W;
    st[4] = nh[0]; st[5] = nh[1]; st[6] = nh[2];
    for (int i = 0; i < 2; ++i)
        for (int d = 0; d < 3; ++d) st[7 + 3 * i + d] = b[i].pos[d] - com[d];
    return BSN_OK;
}

extern "C" bsn_status bsn_kepler_update(bsn_bh* b, const double st[13], double t) {
    if (!b || !st) return BSN_ERR_ARG;
    double th = st[3] * t, c = std::cos(th), s = std::sin(th);
    double nx = st[4], ny = st[5], nz = st[6], W = st[3];
    for (int i = 0; i < 2; ++i) {
        double rx0 = st[7 + 3 * i], ry0 = st[8 + 3 * i], rz0 = st[9 + 3 * i];
        double nd = nx * rx0 + ny * ry0 + nz * rz0;
        double kx = ny * rz0 - nz * ry0, ky = nz * rx0 - nx * rz0, kz = nx * ry0 - ny * rx0;
        double rx = rx0 * c + kx * s + nx * nd * (1.0 - c);
        double ry = ry0 * c + ky * s + ny * nd * (1.0 - c);
        double rz = rz0 * c + kz * s + nz * nd * (1.0 - c);
        b[i].pos[0] = st[0] + rx; b[i].pos[1] = st[1] + ry; b[i].pos[2] = st[2] + rz;
        b[i].vel[0] = W * (ny * rz - nz * ry);
        b[i].vel[1] = W * (nz * rx - nx * rz);
        b[i].vel[2] = W * (nx * ry - ny * rx);
    }
    return BSN_OK;
}

// coupled_step! (scripts/run_sn50_fiducial.jl:756-818)
extern "C" bsn_status bsn_coupled_step_f64(bsn_ctx* ctx, double* U, bsn_bh* bhs, int nbh, double dt, double t, int nx,
                                           int ny, int nz, double dx, double x0, double y0, double z0, double gamma,
                                           double f_sink, double rho_floor, double P_floor, int torque_free,
                                           int self_gravity, double t_bh2_sink_on, double rho_sink_min,
                                           int evolve_orbit, double* Fgas_out) {
    BSN_TRY(check_dims(ctx, nx, ny, nz));
    if (!U || (nbh > 0 && !bhs)) return set_err(ctx, BSN_ERR_ARG, "null argument");
    if (nbh > f64::MAXBH) return set_err(ctx, BSN_ERR_UNSUPPORTED, "at most %d black holes", f64::MAXBH);
    int nsink = (t < t_bh2_sink_on) ? std::min(1, nbh) : nbh;
    std::vector<double> Fg(3 * std::max(nbh, 1), 0.0);
    for (int i = 0; i < nbh; ++i) {
        BSN_TRY(gas_force(ctx, U, nx, ny, nz, dx, dx, dx, bhs[i], x0, y0, z0, &Fg[3 * i]));
        double* F = &Fg[3 * i];
        bool fin = std::isfinite(F[0]) && std::isfinite(F[1]) && std::isfinite(F[2]);
        if (!fin || std::sqrt(F[0] * F[0] + F[1] * F[1] + F[2] * F[2]) > 1e3) F[0] = F[1] = F[2] = 0.0;
    }
    if (evolve_orbit && nbh > 0) {
        bool ok = true;
        for (int i = 0; i < nbh; ++i)
            for (int d = 0; d < 3; ++d) ok = ok && std::isfinite(bhs[i].pos[d]) && std::isfinite(bhs[i].vel[d]);
        if (ok) BSN_TRY(bsn_nbody_step(bhs, nbh, dt, Fg.data()));
    }
    f64::StageArgs A;
    stage_args_init(A, nx, ny, nz, dx, dx, dx, gamma, BSN_BC_OUTFLOW, rho_floor, P_floor);
    A.stiff_guard = 1;
    A.x0 = x0; A.y0 = y0; A.z0 = z0;
    if (nbh > 0) {
        BSN_TRY(fill_bh(ctx, bhs, nbh, A.bh));
        A.use_bh = 1;
    }
    if (nsink > 0) {
        BSN_TRY(fill_sink(ctx, bhs, nsink, f_sink, torque_free, rho_sink_min, A.sk));
        A.use_sink = 1;
    }
    if (self_gravity) {
        BSN_TRY(f64_rk3_selfgrav(ctx, A, U, dt));
    } else {
        BSN_TRY(f64_rk3(ctx, A, U, dt, nullptr, nullptr, nullptr));
    }
    for (int i = 0; i < nsink; ++i)
        BSN_TRY(accrete(ctx, &bhs[i], U, nx, ny, nz, dx, dx, dx, x0, y0, z0, dt, f_sink, rho_sink_min));
    if (Fgas_out)
        for (int i = 0; i < 3 * nbh; ++i) Fgas_out[i] = Fg[i];
    return BSN_OK;
}
