/*
 * bsn_oracle.cpp -- CPU FP64 oracle (TEST INFRASTRUCTURE ONLY; see bsn_oracle.h).
 *
 * Each function restates one reference function and cites it.  Build flags
 * (-O2 -ffp-contract=off -fno-fast-math) keep IEEE-754 double arithmetic in the
 * order written.  OpenMP parallelises only loops whose iterations are
 * independent and whose per-cell arithmetic is unchanged; every reduction that
 * the reference sums sequentially is summed sequentially here.
 */
#include "bsn_oracle.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "hydro.inc"


/* src/euler3d.jl:275-316 */
extern "C" void orc_sedov_ic_3d(double* U, int nx, int ny, int nz, double dx, double dy, double dz, double g,
                                double E_blast, double r_inject, double rho_bg, double P_floor,
                                double x_offset, double y_offset, double z_offset) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    double r_inj = r_inject > 0.0 ? r_inject : 2.5 * jmin(jmin(dx, dy), dz);
    std::memset(U, 0, sizeof(double) * I.size());
    double E_bg = P_floor / (g - 1.0);
    for (int k = ng + 1; k <= ng + nz; ++k) for (int j = ng + 1; j <= ng + ny; ++j)
        for (int i = ng + 1; i <= ng + nx; ++i) { U[I(1, i, j, k)] = rho_bg; U[I(5, i, j, k)] = E_bg; }
    double V_inj = 0.0;
    for (int k = ng + 1; k <= ng + nz; ++k) for (int j = ng + 1; j <= ng + ny; ++j)
        for (int i = ng + 1; i <= ng + nx; ++i) {
            double xc = ((double)(i - ng) - 0.5) * dx + x_offset;
            double yc = ((double)(j - ng) - 0.5) * dy + y_offset;
            double zc = ((double)(k - ng) - 0.5) * dz + z_offset;
            double r = std::sqrt(sq(xc) + sq(yc) + sq(zc));
            if (r <= r_inj) V_inj += dx * dy * dz;
        }
    double dE_cell = (V_inj > 0.0) ? E_blast * (g - 1.0) / V_inj : 0.0;
    for (int k = ng + 1; k <= ng + nz; ++k) for (int j = ng + 1; j <= ng + ny; ++j)
        for (int i = ng + 1; i <= ng + nx; ++i) {
            double xc = ((double)(i - ng) - 0.5) * dx + x_offset;
            double yc = ((double)(j - ng) - 0.5) * dy + y_offset;
            double zc = ((double)(k - ng) - 0.5) * dz + z_offset;
            double r = std::sqrt(sq(xc) + sq(yc) + sq(zc));
            if (r <= r_inj) U[I(5, i, j, k)] += dE_cell;
        }
}

/* ------------------------------------------------------------------------- */
/* src/BinarySupernova.jl:159 */
extern "C" double orc_r_sink(const orc_bh* bh) {
    return jmax(6.0 * bh->mass / sq(bh->c_code), bh->r_floor);
}
/* src/BinarySupernova.jl:167-171 */
extern "C" double orc_t_sink(const orc_bh* bh, double f_sink) {
    double rs = orc_r_sink(bh);
    double v_ff = std::sqrt(2.0 * bh->mass / rs);
    return f_sink * rs / v_ff;
}

/* src/gpu_kernels.jl:199-230 via src/gravity_bh.jl:58-78.  The _slab forms
 * take a z-slab of a larger grid whose first active plane is global plane
 * kofs (0-based): cell centres use the global index, z0 + (kofs + kk - 0.5) dz,
 * so every cell takes the undivided grid's arithmetic. */
extern "C" void orc_add_bh_gravity_source_slab(double* dU, const double* U, int nx, int ny, int nz,
                                               double dx, double dy, double dz, const orc_bh* bhs, int nbh,
                                               double x0, double y0, double z0, int kofs) {
    Idx I(nx, ny, nz);
    const int ng = NG;
#pragma omp parallel for schedule(static)
    for (int kk = 1; kk <= nz; ++kk)
        for (int jj = 1; jj <= ny; ++jj)
            for (int ii = 1; ii <= nx; ++ii) {
                int i = ii + ng, j = jj + ng, k = kk + ng;
                double xc = x0 + ((double)ii - 0.5) * dx;
                double yc = y0 + ((double)jj - 0.5) * dy;
                double zc = z0 + ((double)(kofs + kk) - 0.5) * dz;
                double r = U[I(1, i, j, k)];
                double vx = U[I(2, i, j, k)] / r, vy = U[I(3, i, j, k)] / r, vz = U[I(4, i, j, k)] / r;
                double ax = 0.0, ay = 0.0, az = 0.0;
                for (int n = 0; n < nbh; ++n) {
                    double ddx = xc - bhs[n].pos[0], ddy = yc - bhs[n].pos[1], ddz = zc - bhs[n].pos[2];
                    double r2 = sq(ddx) + sq(ddy) + sq(ddz) + sq(bhs[n].eps);
                    double r3 = r2 * std::sqrt(r2);
                    double fac = -bhs[n].mass / r3;
                    ax += fac * ddx; ay += fac * ddy; az += fac * ddz;
                }
                dU[I(2, i, j, k)] += r * ax;
                dU[I(3, i, j, k)] += r * ay;
                dU[I(4, i, j, k)] += r * az;
                dU[I(5, i, j, k)] += r * (vx * ax + vy * ay + vz * az);
            }
}

extern "C" void orc_add_bh_gravity_source(double* dU, const double* U, int nx, int ny, int nz,
                                          double dx, double dy, double dz, const orc_bh* bhs, int nbh,
                                          double x0, double y0, double z0) {
    orc_add_bh_gravity_source_slab(dU, U, nx, ny, nz, dx, dy, dz, bhs, nbh, x0, y0, z0, 0);
}

/* src/gravity_bh.jl:91-113 (the _slab form: see orc_add_bh_gravity_source_slab) */
extern "C" void orc_gas_force_on_bh_slab(const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                                         const orc_bh* bh, double x0, double y0, double z0, int kofs,
                                         double out[3]) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    double dV = dx * dy * dz;
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        double xc = x0 + ((double)i - 0.5) * dx;
        double yc = y0 + ((double)j - 0.5) * dy;
        double zc = z0 + ((double)(kofs + k) - 0.5) * dz;
        double ddx = xc - bh->pos[0], ddy = yc - bh->pos[1], ddz = zc - bh->pos[2];
        double r2 = sq(ddx) + sq(ddy) + sq(ddz) + sq(bh->eps);
        double r3 = r2 * std::sqrt(r2);
        double fac = bh->mass / r3 * U[I(1, ng + i, ng + j, ng + k)] * dV;
        Fx += fac * ddx; Fy += fac * ddy; Fz += fac * ddz;
    }
    out[0] = Fx; out[1] = Fy; out[2] = Fz;
}

extern "C" void orc_gas_force_on_bh(const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                                    const orc_bh* bh, double x0, double y0, double z0, double out[3]) {
    orc_gas_force_on_bh_slab(U, nx, ny, nz, dx, dy, dz, bh, x0, y0, z0, 0, out);
}

/* src/gpu_kernels.jl:238-284 via src/sinks.jl:32-59 (the _slab form: see
 * orc_add_bh_gravity_source_slab) */
extern "C" void orc_add_sink_sources_slab(double* dU, const double* U, int nx, int ny, int nz,
                                          double dx, double dy, double dz, const orc_bh* bhs, int nbh,
                                          double x0, double y0, double z0, double f_sink, int torque_free,
                                          double rho_sink_min, int kofs) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    std::vector<double> rs(nbh), ts(nbh);
    for (int n = 0; n < nbh; ++n) { rs[n] = orc_r_sink(&bhs[n]); ts[n] = orc_t_sink(&bhs[n], f_sink); }
#pragma omp parallel for schedule(static)
    for (int kk = 1; kk <= nz; ++kk)
        for (int jj = 1; jj <= ny; ++jj)
            for (int ii = 1; ii <= nx; ++ii) {
                int i = ii + ng, j = jj + ng, k = kk + ng;
                double xc = x0 + ((double)ii - 0.5) * dx;
                double yc = y0 + ((double)jj - 0.5) * dy;
                double zc = z0 + ((double)(kofs + kk) - 0.5) * dz;
                double r = U[I(1, i, j, k)];
                double mx = U[I(2, i, j, k)], my = U[I(3, i, j, k)], mz = U[I(4, i, j, k)];
                double E = U[I(5, i, j, k)];
                if (!(r > rho_sink_min)) continue;
                for (int n = 0; n < nbh; ++n) {
                    double ddx = xc - bhs[n].pos[0], ddy = yc - bhs[n].pos[1], ddz = zc - bhs[n].pos[2];
                    double rr = std::sqrt(sq(ddx) + sq(ddy) + sq(ddz));
                    if (rr < rs[n]) {
                        double t = ts[n];
                        dU[I(1, i, j, k)] -= r / t;
                        if (torque_free) {
                            double rx = ddx / rr, ry = ddy / rr, rz = ddz / rr;
                            double vx = mx / r, vy = my / r, vz = mz / r;
                            double vrx = vx - bhs[n].vel[0], vry = vy - bhs[n].vel[1], vrz = vz - bhs[n].vel[2];
                            double v_r = vrx * rx + vry * ry + vrz * rz;
                            double e_int = E / r - 0.5 * (sq(vx) + sq(vy) + sq(vz));
                            dU[I(2, i, j, k)] -= r * v_r * rx / t;
                            dU[I(3, i, j, k)] -= r * v_r * ry / t;
                            dU[I(4, i, j, k)] -= r * v_r * rz / t;
                            dU[I(5, i, j, k)] -= (0.5 * r * sq(v_r) + r * e_int) / t;
                        } else {
                            dU[I(2, i, j, k)] -= mx / t;
                            dU[I(3, i, j, k)] -= my / t;
                            dU[I(4, i, j, k)] -= mz / t;
                            dU[I(5, i, j, k)] -= E / t;
                        }
                    }
                }
            }
}

extern "C" void orc_add_sink_sources(double* dU, const double* U, int nx, int ny, int nz,
                                     double dx, double dy, double dz, const orc_bh* bhs, int nbh,
                                     double x0, double y0, double z0, double f_sink, int torque_free,
                                     double rho_sink_min) {
    orc_add_sink_sources_slab(dU, U, nx, ny, nz, dx, dy, dz, bhs, nbh, x0, y0, z0, f_sink, torque_free,
                              rho_sink_min, 0);
}

/* src/sinks.jl:74-109 */
extern "C" void orc_accrete(orc_bh* bh, const double* U, int nx, int ny, int nz, double dx, double dy,
                            double dz, double x0, double y0, double z0, double dt, double f_sink,
                            double rho_sink_min) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    double rs = orc_r_sink(bh), ts = orc_t_sink(bh, f_sink);
    double dV = dx * dy * dz;
    double dm = 0.0, dPx = 0.0, dPy = 0.0, dPz = 0.0;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        double xc = x0 + ((double)i - 0.5) * dx;
        double yc = y0 + ((double)j - 0.5) * dy;
        double zc = z0 + ((double)k - 0.5) * dz;
        double r = std::sqrt(sq(xc - bh->pos[0]) + sq(yc - bh->pos[1]) + sq(zc - bh->pos[2]));
        if (r >= rs) continue;
        if (U[I(1, ng + i, ng + j, ng + k)] <= rho_sink_min) continue;
        double rate = dV / ts * dt;
        dm += U[I(1, ng + i, ng + j, ng + k)] * rate;
        dPx += U[I(2, ng + i, ng + j, ng + k)] * rate;
        dPy += U[I(3, ng + i, ng + j, ng + k)] * rate;
        dPz += U[I(4, ng + i, ng + j, ng + k)] * rate;
    }
    if (dm > 0.0) {
        double M_new = bh->mass + dm;
        bh->vel[0] = (bh->mass * bh->vel[0] + dPx) / M_new;
        bh->vel[1] = (bh->mass * bh->vel[1] + dPy) / M_new;
        bh->vel[2] = (bh->mass * bh->vel[2] + dPz) / M_new;
        bh->mass = M_new;
    }
}

/* The terms accrete! (src/sinks.jl:74-109) adds, for the cells of the
 * global active box [ilo,ihi] x [jlo,jhi] x [klo,khi] (0-based, inclusive)
 * that lie in this z-slab (global planes kofs .. kofs + nz - 1), in the
 * reference's (k, j, i) loop order: {rho, mx, my, mz} * rate for a cell in
 * the sink sphere with rho > rho_sink_min, zeros for any other cell (adding
 * +0.0 leaves the sequential sums as skipping the cell does).  Returns the
 * number of cells written (4 doubles each). */
extern "C" long orc_sink_terms_slab(const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                                    double x0, double y0, double z0, int kofs, const orc_bh* bh, double rate,
                                    double rho_sink_min, int ilo, int ihi, int jlo, int jhi, int klo, int khi,
                                    double* out) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    double rs = orc_r_sink(bh);
    long n = 0;
    int k_lo = std::max(klo, kofs), k_hi = std::min(khi, kofs + nz - 1);
    for (int kg = k_lo; kg <= k_hi; ++kg) for (int j = jlo; j <= jhi; ++j) for (int i = ilo; i <= ihi; ++i) {
        double xc = x0 + ((double)(i + 1) - 0.5) * dx;
        double yc = y0 + ((double)(j + 1) - 0.5) * dy;
        double zc = z0 + ((double)(kg + 1) - 0.5) * dz;
        double r = std::sqrt(sq(xc - bh->pos[0]) + sq(yc - bh->pos[1]) + sq(zc - bh->pos[2]));
        double* o = out + 4 * n++;
        o[0] = o[1] = o[2] = o[3] = 0.0;
        int k = kg - kofs;
        if (r >= rs) continue;
        if (U[I(1, ng + 1 + i, ng + 1 + j, ng + 1 + k)] <= rho_sink_min) continue;
        for (int q = 0; q < 4; ++q) o[q] = U[I(1 + q, ng + 1 + i, ng + 1 + j, ng + 1 + k)] * rate;
    }
    return n;
}

/* src/nbody.jl:24-56 */
static void nbody_rhs(double (*dpos)[3], double (*dvel)[3], const orc_bh* bhs, int n, const double* Fg) {
    for (int i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) dpos[i][d] = bhs[i].vel[d];
        double a[3];
        for (int d = 0; d < 3; ++d) a[d] = Fg[3 * i + d] / bhs[i].mass;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            double dx = bhs[j].pos[0] - bhs[i].pos[0];
            double dy = bhs[j].pos[1] - bhs[i].pos[1];
            double dz = bhs[j].pos[2] - bhs[i].pos[2];
            double r2 = sq(dx) + sq(dy) + sq(dz) + sq(bhs[j].eps);
            double r3 = r2 * std::sqrt(r2);
            double fac = bhs[j].mass / r3;
            a[0] = a[0] + fac * dx; a[1] = a[1] + fac * dy; a[2] = a[2] + fac * dz;
        }
        for (int d = 0; d < 3; ++d) dvel[i][d] = a[d];
    }
}

/* src/nbody.jl:74-104 */
extern "C" void orc_nbody_step(orc_bh* bhs, int n, double dt, const double* Fg) {
    std::vector<double> p0(3 * n), v0(3 * n), p1(3 * n), v1(3 * n), p2(3 * n), v2(3 * n);
    std::vector<double> dp(3 * n), dv(3 * n);
    auto DP = reinterpret_cast<double (*)[3]>(dp.data());
    auto DV = reinterpret_cast<double (*)[3]>(dv.data());
    for (int i = 0; i < n; ++i) for (int d = 0; d < 3; ++d) { p0[3*i+d] = bhs[i].pos[d]; v0[3*i+d] = bhs[i].vel[d]; }
    nbody_rhs(DP, DV, bhs, n, Fg);
    for (int i = 0; i < n; ++i) for (int d = 0; d < 3; ++d) {
        p1[3*i+d] = p0[3*i+d] + dt * DP[i][d];
        v1[3*i+d] = v0[3*i+d] + dt * DV[i][d];
    }
    for (int i = 0; i < n; ++i) for (int d = 0; d < 3; ++d) { bhs[i].pos[d] = p1[3*i+d]; bhs[i].vel[d] = v1[3*i+d]; }
    nbody_rhs(DP, DV, bhs, n, Fg);
    for (int i = 0; i < n; ++i) for (int d = 0; d < 3; ++d) {
        p2[3*i+d] = 0.75 * p0[3*i+d] + 0.25 * (p1[3*i+d] + dt * DP[i][d]);
        v2[3*i+d] = 0.75 * v0[3*i+d] + 0.25 * (v1[3*i+d] + dt * DV[i][d]);
    }
    for (int i = 0; i < n; ++i) for (int d = 0; d < 3; ++d) { bhs[i].pos[d] = p2[3*i+d]; bhs[i].vel[d] = v2[3*i+d]; }
    nbody_rhs(DP, DV, bhs, n, Fg);
    for (int i = 0; i < n; ++i) for (int d = 0; d < 3; ++d) {
        bhs[i].pos[d] = (1.0 / 3.0) * p0[3*i+d] + (2.0 / 3.0) * (p2[3*i+d] + dt * DP[i][d]);
        bhs[i].vel[d] = (1.0 / 3.0) * v0[3*i+d] + (2.0 / 3.0) * (v2[3*i+d] + dt * DV[i][d]);
    }
}

/* src/kepler_orbit.jl:63-111 */
extern "C" int orc_kepler_init(const orc_bh* bhs, const double com[3], const double* nhat, double Omega,
                               double st[13]) {
    double dx = bhs[0].pos[0] - bhs[1].pos[0], dy = bhs[0].pos[1] - bhs[1].pos[1],
           dz = bhs[0].pos[2] - bhs[1].pos[2];
    double a = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (!(a > 0)) return -1;
    double rx1 = bhs[0].pos[0] - com[0], ry1 = bhs[0].pos[1] - com[1], rz1 = bhs[0].pos[2] - com[2];
    double vx1 = bhs[0].vel[0], vy1 = bhs[0].vel[1], vz1 = bhs[0].vel[2];
    double nh[3];
    if (!nhat) {
        double Lx = ry1 * vz1 - rz1 * vy1, Ly = rz1 * vx1 - rx1 * vz1, Lz = rx1 * vy1 - ry1 * vx1;
        double Lm = std::sqrt(Lx * Lx + Ly * Ly + Lz * Lz);
        if (!(Lm > 0)) return -2;
        nh[0] = Lx / Lm; nh[1] = Ly / Lm; nh[2] = Lz / Lm;
    } else {
        double nm = std::sqrt(sq(nhat[0]) + sq(nhat[1]) + sq(nhat[2]));
        if (!(std::fabs(nm - 1.0) < 1e-10)) return -3;
        nh[0] = nhat[0]; nh[1] = nhat[1]; nh[2] = nhat[2];
    }
    double W;
    if (!(Omega > 0)) {
        double Rmag = std::sqrt(rx1 * rx1 + ry1 * ry1 + rz1 * rz1);
        double vmag = std::sqrt(vx1 * vx1 + vy1 * vy1 + vz1 * vz1);
        if (!(Rmag > 0) || !(vmag > 0)) return -4;
        W = vmag / Rmag;
    } else {
        W = Omega;
    }
    st[0] = com[0]; st[1] = com[1]; st[2] = com[2]; st[3] = W;
    st[4] = nh[0]; st[5] = nh[1]; st[6] = nh[2];
    for (int i = 0; i < 2; ++i)
        for (int d = 0; d < 3; ++d) st[7 + 3 * i + d] = bhs[i].pos[d] - com[d];
    return 0;
}

/* src/kepler_orbit.jl:124-150 */
extern "C" void orc_kepler_update(orc_bh* bhs, const double st[13], double t) {
    double th = st[3] * t;
    double c = std::cos(th), s = std::sin(th);
    double nx = st[4], ny = st[5], nz = st[6];
    double cx = st[0], cy = st[1], cz = st[2];
    double W = st[3];
    for (int i = 0; i < 2; ++i) {
        double rx0 = st[7 + 3 * i], ry0 = st[8 + 3 * i], rz0 = st[9 + 3 * i];
        double ndotr = nx * rx0 + ny * ry0 + nz * rz0;
        double kx = ny * rz0 - nz * ry0, ky = nz * rx0 - nx * rz0, kz = nx * ry0 - ny * rx0;
        double rx = rx0 * c + kx * s + nx * ndotr * (1.0 - c);
        double ry = ry0 * c + ky * s + ny * ndotr * (1.0 - c);
        double rz = rz0 * c + kz * s + nz * ndotr * (1.0 - c);
        bhs[i].pos[0] = cx + rx; bhs[i].pos[1] = cy + ry; bhs[i].pos[2] = cz + rz;
        bhs[i].vel[0] = W * (ny * rz - nz * ry);
        bhs[i].vel[1] = W * (nz * rx - nx * rz);
        bhs[i].vel[2] = W * (nx * ry - ny * rx);
    }
}

/* ------------------------------------------------------------------------- */
/* FFT: iterative radix-2 for powers of two, direct DFT otherwise.  Stands in
 * for FFTW/cuFFT behind AbstractFFTs fft/ifft (src/self_gravity.jl:73);
 * inverse includes the 1/N normalisation as ifft does. */
namespace {
void fft1d(double* re, double* im, int n, long stride, int inverse, std::vector<double>& tr,
           std::vector<double>& ti) {
    tr.resize(n); ti.resize(n);
    for (int t = 0; t < n; ++t) { tr[t] = re[t * stride]; ti[t] = im[t * stride]; }
    double sgn = inverse ? 1.0 : -1.0;
    if ((n & (n - 1)) == 0) {
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) { std::swap(tr[i], tr[j]); std::swap(ti[i], ti[j]); }
        }
        for (int len = 2; len <= n; len <<= 1) {
            int half = len >> 1;
            for (int s = 0; s < n; s += len)
                for (int m = 0; m < half; ++m) {
                    double ang = sgn * 2.0 * M_PI * (double)m / (double)len;
                    double wr = std::cos(ang), wi = std::sin(ang);
                    double ur = tr[s + m], ui = ti[s + m];
                    double xr = tr[s + m + half], xi = ti[s + m + half];
                    double vr = xr * wr - xi * wi, vi = xr * wi + xi * wr;
                    tr[s + m] = ur + vr; ti[s + m] = ui + vi;
                    tr[s + m + half] = ur - vr; ti[s + m + half] = ui - vi;
                }
        }
    } else {
        std::vector<double> orr(n), oi(n);
        for (int kf = 0; kf < n; ++kf) {
            double sr = 0.0, si = 0.0;
            for (int t = 0; t < n; ++t) {
                long p = ((long)kf * t) % n;
                double ang = sgn * 2.0 * M_PI * (double)p / (double)n;
                double wr = std::cos(ang), wi = std::sin(ang);
                sr += tr[t] * wr - ti[t] * wi;
                si += tr[t] * wi + ti[t] * wr;
            }
            orr[kf] = sr; oi[kf] = si;
        }
        tr = orr; ti = oi;
    }
    double sc = inverse ? 1.0 / (double)n : 1.0;
    for (int t = 0; t < n; ++t) { re[t * stride] = tr[t] * sc; im[t * stride] = ti[t] * sc; }
}
}  // namespace

extern "C" void orc_fft3d(double* re, double* im, int n1, int n2, int n3, int inverse) {
    /* column-major (n1 fastest) */
#pragma omp parallel
    {
        std::vector<double> tr, ti;
#pragma omp for schedule(static)
        for (long l = 0; l < (long)n2 * n3; ++l) fft1d(re + l * n1, im + l * n1, n1, 1, inverse, tr, ti);
#pragma omp for schedule(static)
        for (long l = 0; l < (long)n1 * n3; ++l) {
            long a = l % n1, c = l / n1;
            fft1d(re + a + c * (long)n1 * n2, im + a + c * (long)n1 * n2, n2, n1, inverse, tr, ti);
        }
#pragma omp for schedule(static)
        for (long l = 0; l < (long)n1 * n2; ++l)
            fft1d(re + l, im + l, n3, (long)n1 * n2, inverse, tr, ti);
    }
}

/* src/self_gravity.jl:35-76 */
extern "C" void orc_solve_poisson_isolated(const double* rho, int nx, int ny, int nz,
                                           double dx, double dy, double dz, double* phi) {
    int Nx = 2 * nx, Ny = 2 * ny, Nz = 2 * nz;
    double dV = dx * dy * dz;
    double eps2 = std::pow(dx * dy * dz, 2.0 / 3.0);
    long N = (long)Nx * Ny * Nz;
    std::vector<double> Kr(N), Ki(N, 0.0), Rr(N, 0.0), Ri(N, 0.0);
    for (int k = 1; k <= Nz; ++k) for (int j = 1; j <= Ny; ++j) for (int i = 1; i <= Nx; ++i) {
        double fi = (double)(i <= nx ? i - 1 : i - 1 - Nx);
        double fj = (double)(j <= ny ? j - 1 : j - 1 - Ny);
        double fk = (double)(k <= nz ? k - 1 : k - 1 - Nz);
        double r2 = sq(fi * dx) + sq(fj * dy) + sq(fk * dz);
        Kr[(i - 1) + (long)Nx * ((j - 1) + (long)Ny * (k - 1))] = -1.0 / std::sqrt(r2 + eps2);
    }
    for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i)
        Rr[i + (long)Nx * (j + (long)Ny * k)] = rho[i + (long)nx * (j + (long)ny * k)];
    orc_fft3d(Kr.data(), Ki.data(), Nx, Ny, Nz, 0);
    orc_fft3d(Rr.data(), Ri.data(), Nx, Ny, Nz, 0);
    for (long t = 0; t < N; ++t) {
        double ar = Kr[t], ai = Ki[t], br = Rr[t], bi = Ri[t];
        Rr[t] = ar * br - ai * bi;
        Ri[t] = ar * bi + ai * br;
    }
    orc_fft3d(Rr.data(), Ri.data(), Nx, Ny, Nz, 1);
    for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i)
        phi[i + (long)nx * (j + (long)ny * k)] = Rr[i + (long)Nx * (j + (long)Ny * k)] * dV;
}

/* src/gpu_kernels.jl:291-319 (via src/fmr_gravity.jl:146-156) */
extern "C" void orc_sg_gradient(double* dU, const double* U, const double* phi, int nx, int ny, int nz,
                                double dx, double dy, double dz) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    double inv2dx = 0.5 / dx, inv2dy = 0.5 / dy, inv2dz = 0.5 / dz;
    auto P = [&](int a, int b, int c) { return phi[(a - 1) + (long)nx * ((b - 1) + (long)ny * (c - 1))]; };
#pragma omp parallel for schedule(static)
    for (int kk = 1; kk <= nz; ++kk)
        for (int jj = 1; jj <= ny; ++jj)
            for (int ii = 1; ii <= nx; ++ii) {
                int i = ii + ng, j = jj + ng, k = kk + ng;
                double r = U[I(1, i, j, k)];
                double rvx = U[I(2, i, j, k)], rvy = U[I(3, i, j, k)], rvz = U[I(4, i, j, k)];
                int ip = std::min(ii + 1, nx), im = std::max(ii - 1, 1);
                int jp = std::min(jj + 1, ny), jm = std::max(jj - 1, 1);
                int kp = std::min(kk + 1, nz), km = std::max(kk - 1, 1);
                double fxfac = ip > im ? inv2dx : 2.0 * inv2dx;
                double fyfac = jp > jm ? inv2dy : 2.0 * inv2dy;
                double fzfac = kp > km ? inv2dz : 2.0 * inv2dz;
                double gx = (P(ip, jj, kk) - P(im, jj, kk)) * fxfac;
                double gy = (P(ii, jp, kk) - P(ii, jm, kk)) * fyfac;
                double gz = (P(ii, jj, kp) - P(ii, jj, km)) * fzfac;
                double vdotg = (rvx * gx + rvy * gy + rvz * gz) / r;
                dU[I(2, i, j, k)] -= r * gx;
                dU[I(3, i, j, k)] -= r * gy;
                dU[I(4, i, j, k)] -= r * gz;
                dU[I(5, i, j, k)] -= r * vdotg;
            }
}

/* src/self_gravity.jl:93-115 */
extern "C" void orc_add_self_gravity_source(double* dU, const double* U, int nx, int ny, int nz,
                                            double dx, double dy, double dz) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    std::vector<double> rho((long)nx * ny * nz), phi((long)nx * ny * nz);
    for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i)
        rho[i + (long)nx * (j + (long)ny * k)] = U[I(1, ng + 1 + i, ng + 1 + j, ng + 1 + k)];
    orc_solve_poisson_isolated(rho.data(), nx, ny, nz, dx, dy, dz, phi.data());
    orc_sg_gradient(dU, U, phi.data(), nx, ny, nz, dx, dy, dz);
}

/* scripts/run_sn50_fiducial.jl:756-818 (coupled_step!).  evolve_orbit=1 runs
 * nbody_step!; 0 leaves BHs as given (caller applies kepler_update!). */
extern "C" void orc_coupled_step(double* U, double* Un, double* dU, double* Fx, double* Fy, double* Fz,
                                 orc_bh* bhs, int nbh, double dt, double t, int nx, int ny, int nz,
                                 double dx, double x0, double y0, double z0, double g,
                                 double f_sink, double rho_floor, double P_floor, int torque_free,
                                 int self_gravity, double t_bh2_sink_on, double rho_sink_min,
                                 int evolve_orbit, double* Fgas) {
    Idx I(nx, ny, nz);
    long n = I.size();
    int nsink = (t < t_bh2_sink_on) ? std::min(1, nbh) : nbh;
    for (int i = 0; i < nbh; ++i) {
        orc_gas_force_on_bh(U, nx, ny, nz, dx, dx, dx, &bhs[i], x0, y0, z0, Fgas + 3 * i);
        double* F = Fgas + 3 * i;
        bool fin = std::isfinite(F[0]) && std::isfinite(F[1]) && std::isfinite(F[2]);
        if (!fin || std::sqrt(sq(F[0]) + sq(F[1]) + sq(F[2])) > 1e3) { F[0] = F[1] = F[2] = 0.0; }
    }
    if (evolve_orbit) {
        bool ok = true;
        for (int i = 0; i < nbh; ++i)
            for (int d = 0; d < 3; ++d) ok = ok && std::isfinite(bhs[i].pos[d]) && std::isfinite(bhs[i].vel[d]);
        if (ok) orc_nbody_step(bhs, nbh, dt, Fgas);
    }
    std::memcpy(Un, U, sizeof(double) * n);
    for (int stage = 0; stage < 3; ++stage) {
        orc_euler3d_rhs(dU, Fx, Fy, Fz, U, nx, ny, nz, dx, dx, dx, g, 0, rho_floor, P_floor, 1);
        orc_add_bh_gravity_source(dU, U, nx, ny, nz, dx, dx, dx, bhs, nbh, x0, y0, z0);
        if (self_gravity) orc_add_self_gravity_source(dU, U, nx, ny, nz, dx, dx, dx);
        orc_add_sink_sources(dU, U, nx, ny, nz, dx, dx, dx, bhs, nsink, x0, y0, z0, f_sink, torque_free,
                             rho_sink_min);
        if (stage == 0) combine1(U, Un, dU, dt, n);
        else if (stage == 1) combine2(U, Un, dU, dt, n);
        else combine3(U, Un, dU, dt, n);
        orc_apply_floors(U, nx, ny, nz, rho_floor, P_floor, g);
    }
    for (int i = 0; i < nsink; ++i)
        orc_accrete(&bhs[i], U, nx, ny, nz, dx, dx, dx, x0, y0, z0, dt, f_sink, rho_sink_min);
}

/* ------------------------------------------------------------------------- */
/* src/fmr3d.jl:32-46; w is (ratio x 5) column-major: w[s + ratio*j] */
extern "C" void orc_lag5_weights(int ratio, double* w) {
    const double nodes[5] = {-2.0, -1.0, 0.0, 1.0, 2.0};
    for (int s = 0; s < ratio; ++s) {
        double t = ((double)s + 0.5 - (double)ratio / 2.0) / (double)ratio;
        for (int j = 0; j < 5; ++j) {
            double wj = 1.0;
            for (int m = 0; m < 5; ++m)
                if (m != j) wj *= (t - nodes[m]) / (nodes[j] - nodes[m]);
            w[s + ratio * j] = wj;
        }
    }
}

namespace {
/* src/fmr3d.jl:165-170; round(Int, x) is round-half-even. */
inline void coarse_stencil(int ig_f, int c_lo, int ratio, int ng, int* ic0, int* sx) {
    double xi = (double)c_lo - 0.5 + ((double)(ig_f - ng) - 0.5) / (double)ratio;
    int c0 = (int)std::nearbyint(xi);
    int s = (int)std::floor((xi - (double)c0 + 0.5) * (double)ratio);
    if (s < 0) s = 0;
    if (s > ratio - 1) s = ratio - 1;
    *ic0 = c0; *sx = s;
}

struct Fmr {
    const orc_fmr* G;
    std::vector<double> w;
    Fmr(const orc_fmr* g) : G(g), w(5 * g->ratio) { orc_lag5_weights(g->ratio, w.data()); }
    double W(int s, int j) const { return w[s + G->ratio * j]; }   /* Julia w[s+1, j+1] */
};

/* src/fmr3d.jl:176-198 */
void prolong_cell(double* Uf, const double* Uc, const Fmr& F, int ig_f, int jf, int kf) {
    const orc_fmr* G = F.G;
    const int r = G->ratio, ng = NG;
    Idx Ic(G->ncx, G->ncy, G->ncz), If(G->nfx, G->nfy, G->nfz);
    int ic0, si, jc0, sj, kc0, sk;
    coarse_stencil(ig_f, G->ci_lo, r, ng, &ic0, &si);
    coarse_stencil(jf, G->cj_lo, r, ng, &jc0, &sj);
    coarse_stencil(kf, G->ck_lo, r, ng, &kc0, &sk);
    for (int q = 1; q <= 5; ++q) {
        double val = 0.0;
        for (int di = -2; di <= 2; ++di) {
            int ig_c = ng + ic0 + di;
            double wi = F.W(si, di + 2);
            for (int dj = -2; dj <= 2; ++dj) {
                int jg_c = ng + jc0 + dj;
                double wij = wi * F.W(sj, dj + 2);
                for (int dk = -2; dk <= 2; ++dk) {
                    int kg_c = ng + kc0 + dk;
                    val += wij * F.W(sk, dk + 2) * Uc[Ic(q, ig_c, jg_c, kg_c)];
                }
            }
        }
        Uf[If(q, ig_f, jf, kf)] = val;
    }
}
}  // namespace

/* src/fmr3d.jl:206-214 */
extern "C" void orc_prolong_all(const orc_fmr* G) {
    Fmr F(G);
    int nxt = G->nfx + 2 * NG, nyt = G->nfy + 2 * NG, nzt = G->nfz + 2 * NG;
#pragma omp parallel for schedule(static)
    for (int kf = 1; kf <= nzt; ++kf)
        for (int jf = 1; jf <= nyt; ++jf)
            for (int ig = 1; ig <= nxt; ++ig) prolong_cell(G->Uf, G->Uc, F, ig, jf, kf);
}

/* src/fmr3d.jl:223-255 */
extern "C" void orc_prolong_fine_ghosts(double* Uf, const double* Uc, const orc_fmr* G) {
    Fmr F(G);
    const int ng = NG;
    int nxf = G->nfx, nyf = G->nfy, nzf = G->nfz;
    int nxt = nxf + 2 * ng, nyt = nyf + 2 * ng, nzt = nzf + 2 * ng;
#pragma omp parallel for schedule(static)
    for (int kf = 1; kf <= nzt; ++kf)
        for (int jf = 1; jf <= nyt; ++jf) {
            for (int ig = 1; ig <= ng; ++ig) prolong_cell(Uf, Uc, F, ig, jf, kf);
            for (int ig = ng + nxf + 1; ig <= nxt; ++ig) prolong_cell(Uf, Uc, F, ig, jf, kf);
        }
#pragma omp parallel for schedule(static)
    for (int kf = 1; kf <= nzt; ++kf)
        for (int ig = ng + 1; ig <= ng + nxf; ++ig) {
            for (int jf = 1; jf <= ng; ++jf) prolong_cell(Uf, Uc, F, ig, jf, kf);
            for (int jf = ng + nyf + 1; jf <= nyt; ++jf) prolong_cell(Uf, Uc, F, ig, jf, kf);
        }
#pragma omp parallel for schedule(static)
    for (int jf = ng + 1; jf <= ng + nyf; ++jf)
        for (int ig = ng + 1; ig <= ng + nxf; ++ig) {
            for (int kf = 1; kf <= ng; ++kf) prolong_cell(Uf, Uc, F, ig, jf, kf);
            for (int kf = ng + nzf + 1; kf <= nzt; ++kf) prolong_cell(Uf, Uc, F, ig, jf, kf);
        }
}

/* src/fmr3d.jl:266-285 */
extern "C" void orc_restrict(double* Uc, const double* Uf, const orc_fmr* G) {
    const int r = G->ratio, ng = NG;
    double inv_r3 = 1.0 / (double)(r * r * r);
    Idx Ic(G->ncx, G->ncy, G->ncz), If(G->nfx, G->nfy, G->nfz);
    for (int m = 0; m <= G->ci_hi - G->ci_lo; ++m)
        for (int n = 0; n <= G->cj_hi - G->cj_lo; ++n)
            for (int p = 0; p <= G->ck_hi - G->ck_lo; ++p) {
                int ic = ng + G->ci_lo + m, jc = ng + G->cj_lo + n, kc = ng + G->ck_lo + p;
                for (int q = 1; q <= 5; ++q) {
                    double val = 0.0;
                    for (int sx = 1; sx <= r; ++sx) for (int sy = 1; sy <= r; ++sy) for (int sz = 1; sz <= r; ++sz)
                        val += Uf[If(q, ng + r * m + sx, ng + r * n + sy, ng + r * p + sz)];
                    Uc[Ic(q, ic, jc, kc)] = val * inv_r3;
                }
            }
}

namespace {
struct FluxReg {   /* src/fmr3d.jl:81-96 */
    int nic, njc, nkc;
    std::vector<double> xlo, xhi, ylo, yhi, zlo, zhi;
    FluxReg(int a, int b, int c) : nic(a), njc(b), nkc(c),
        xlo(5L * b * c, 0.0), xhi(5L * b * c, 0.0), ylo(5L * a * c, 0.0), yhi(5L * a * c, 0.0),
        zlo(5L * a * b, 0.0), zhi(5L * a * b, 0.0) {}
};
inline long R3(int q, int a, int b, int ea) { return (long)(q - 1) + 5L * ((long)(a - 1) + (long)ea * (b - 1)); }

/* src/fmr3d.jl:292-326 */
void accumulate_fr_coarse(FluxReg& fr, const double* Fx, const double* Fy, const double* Fz, double weight,
                          double dt, const orc_fmr* G) {
    const int ng = NG;
    double fac = weight * dt;
    Idx I(G->ncx, G->ncy, G->ncz);
    FIdx X(I.nxt + 1, I.nyt, I.nzt), Y(I.nxt, I.nyt + 1, I.nzt), Z(I.nxt, I.nyt, I.nzt + 1);
    for (int kc = G->ck_lo; kc <= G->ck_hi; ++kc) for (int jc = G->cj_lo; jc <= G->cj_hi; ++jc) {
        int ki = kc - G->ck_lo + 1, ji = jc - G->cj_lo + 1;
        for (int q = 1; q <= 5; ++q) {
            fr.xlo[R3(q, ji, ki, fr.njc)] += fac * Fx[X(q, ng + G->ci_lo - 1, ng + jc, ng + kc)];
            fr.xhi[R3(q, ji, ki, fr.njc)] += fac * Fx[X(q, ng + G->ci_hi, ng + jc, ng + kc)];
        }
    }
    for (int kc = G->ck_lo; kc <= G->ck_hi; ++kc) for (int ic = G->ci_lo; ic <= G->ci_hi; ++ic) {
        int ki = kc - G->ck_lo + 1, ii = ic - G->ci_lo + 1;
        for (int q = 1; q <= 5; ++q) {
            fr.ylo[R3(q, ii, ki, fr.nic)] += fac * Fy[Y(q, ng + ic, ng + G->cj_lo - 1, ng + kc)];
            fr.yhi[R3(q, ii, ki, fr.nic)] += fac * Fy[Y(q, ng + ic, ng + G->cj_hi, ng + kc)];
        }
    }
    for (int jc = G->cj_lo; jc <= G->cj_hi; ++jc) for (int ic = G->ci_lo; ic <= G->ci_hi; ++ic) {
        int ji = jc - G->cj_lo + 1, ii = ic - G->ci_lo + 1;
        for (int q = 1; q <= 5; ++q) {
            fr.zlo[R3(q, ii, ji, fr.nic)] += fac * Fz[Z(q, ng + ic, ng + jc, ng + G->ck_lo - 1)];
            fr.zhi[R3(q, ii, ji, fr.nic)] += fac * Fz[Z(q, ng + ic, ng + jc, ng + G->ck_hi)];
        }
    }
}

/* src/fmr3d.jl:331-369 */
void accumulate_fr_fine(FluxReg& fr, const double* Fx, const double* Fy, const double* Fz, double weight,
                        double dt, const orc_fmr* G) {
    const int ng = NG, r = G->ratio;
    double fac = weight * dt / (double)(r * r);
    int nxf = G->nfx, nyf = G->nfy, nzf = G->nfz;
    Idx I(nxf, nyf, nzf);
    FIdx X(I.nxt + 1, I.nyt, I.nzt), Y(I.nxt, I.nyt + 1, I.nzt), Z(I.nxt, I.nyt, I.nzt + 1);
    for (int kf = 1; kf <= nzf; ++kf) for (int jf = 1; jf <= nyf; ++jf) {
        int ki = (kf - 1) / r + 1, ji = (jf - 1) / r + 1;
        for (int q = 1; q <= 5; ++q) {
            fr.xlo[R3(q, ji, ki, fr.njc)] += fac * Fx[X(q, ng, ng + jf, ng + kf)];
            fr.xhi[R3(q, ji, ki, fr.njc)] += fac * Fx[X(q, ng + nxf, ng + jf, ng + kf)];
        }
    }
    for (int kf = 1; kf <= nzf; ++kf) for (int ia = 1; ia <= nxf; ++ia) {
        int ki = (kf - 1) / r + 1, ii = (ia - 1) / r + 1;
        for (int q = 1; q <= 5; ++q) {
            fr.ylo[R3(q, ii, ki, fr.nic)] += fac * Fy[Y(q, ng + ia, ng, ng + kf)];
            fr.yhi[R3(q, ii, ki, fr.nic)] += fac * Fy[Y(q, ng + ia, ng + nyf, ng + kf)];
        }
    }
    for (int jf = 1; jf <= nyf; ++jf) for (int ia = 1; ia <= nxf; ++ia) {
        int ji = (jf - 1) / r + 1, ii = (ia - 1) / r + 1;
        for (int q = 1; q <= 5; ++q) {
            fr.zlo[R3(q, ii, ji, fr.nic)] += fac * Fz[Z(q, ng + ia, ng + jf, ng)];
            fr.zhi[R3(q, ii, ji, fr.nic)] += fac * Fz[Z(q, ng + ia, ng + jf, ng + nzf)];
        }
    }
}

/* src/fmr3d.jl:379-422 */
void bc_correct(const orc_fmr* G, const FluxReg& fc, const FluxReg& ff) {
    const int ng = NG;
    Idx I(G->ncx, G->ncy, G->ncz);
    double* U = G->Uc;
    int nic = G->ci_hi - G->ci_lo + 1, njc = G->cj_hi - G->cj_lo + 1, nkc = G->ck_hi - G->ck_lo + 1;
    double inv_dx = 1.0 / G->dxc, inv_dy = 1.0 / G->dyc, inv_dz = 1.0 / G->dzc;
    for (int ki = 1; ki <= nkc; ++ki) for (int ji = 1; ji <= njc; ++ji) {
        int jc = G->cj_lo + ji - 1, kc = G->ck_lo + ki - 1;
        for (int q = 1; q <= 5; ++q) {
            double dlo = (fc.xlo[R3(q, ji, ki, njc)] - ff.xlo[R3(q, ji, ki, njc)]) * inv_dx;
            double dhi = (ff.xhi[R3(q, ji, ki, njc)] - fc.xhi[R3(q, ji, ki, njc)]) * inv_dx;
            U[I(q, ng + G->ci_lo - 1, ng + jc, ng + kc)] += dlo;
            U[I(q, ng + G->ci_hi + 1, ng + jc, ng + kc)] += dhi;
        }
    }
    for (int ki = 1; ki <= nkc; ++ki) for (int ii = 1; ii <= nic; ++ii) {
        int ic = G->ci_lo + ii - 1, kc = G->ck_lo + ki - 1;
        for (int q = 1; q <= 5; ++q) {
            double dlo = (fc.ylo[R3(q, ii, ki, nic)] - ff.ylo[R3(q, ii, ki, nic)]) * inv_dy;
            double dhi = (ff.yhi[R3(q, ii, ki, nic)] - fc.yhi[R3(q, ii, ki, nic)]) * inv_dy;
            U[I(q, ng + ic, ng + G->cj_lo - 1, ng + kc)] += dlo;
            U[I(q, ng + ic, ng + G->cj_hi + 1, ng + kc)] += dhi;
        }
    }
    for (int ji = 1; ji <= njc; ++ji) for (int ii = 1; ii <= nic; ++ii) {
        int ic = G->ci_lo + ii - 1, jc = G->cj_lo + ji - 1;
        for (int q = 1; q <= 5; ++q) {
            double dlo = (fc.zlo[R3(q, ii, ji, nic)] - ff.zlo[R3(q, ii, ji, nic)]) * inv_dz;
            double dhi = (ff.zhi[R3(q, ii, ji, nic)] - fc.zhi[R3(q, ii, ji, nic)]) * inv_dz;
            U[I(q, ng + ic, ng + jc, ng + G->ck_lo - 1)] += dlo;
            U[I(q, ng + ic, ng + jc, ng + G->ck_hi + 1)] += dhi;
        }
    }
}

/* src/fmr3d.jl:427-436 */
void fine_rhs(double* dU, double* Fx, double* Fy, double* Fz, double* U, const orc_fmr* G) {
    orc_apply_floors(U, G->nfx, G->nfy, G->nfz, G->rho_floor, G->P_floor, G->gamma);
    Idx I(G->nfx, G->nfy, G->nfz);
    std::memset(Fx, 0, sizeof(double) * 5L * (I.nxt + 1) * I.nyt * I.nzt);
    std::memset(Fy, 0, sizeof(double) * 5L * I.nxt * (I.nyt + 1) * I.nzt);
    std::memset(Fz, 0, sizeof(double) * 5L * I.nxt * I.nyt * (I.nzt + 1));
    orc_weno_fluxes(0, Fx, U, G->nfx, G->nfy, G->nfz, G->gamma);
    orc_weno_fluxes(1, Fy, U, G->nfx, G->nfy, G->nfz, G->gamma);
    orc_weno_fluxes(2, Fz, U, G->nfx, G->nfy, G->nfz, G->gamma);
    orc_flux_divergence(dU, Fx, Fy, Fz, G->nfx, G->nfy, G->nfz, G->dxf, G->dyf, G->dzf);
}
}  // namespace

/* src/fmr_gravity.jl:40-60 */
extern "C" void orc_restrict_density_to_coarse(const orc_fmr* G) {
    const int r = G->ratio, ng = NG;
    double inv_r3 = 1.0 / (double)(r * r * r);
    Idx Ic(G->ncx, G->ncy, G->ncz), If(G->nfx, G->nfy, G->nfz);
    for (int m = 0; m <= G->ci_hi - G->ci_lo; ++m)
        for (int n = 0; n <= G->cj_hi - G->cj_lo; ++n)
            for (int p = 0; p <= G->ck_hi - G->ck_lo; ++p) {
                int ic = ng + G->ci_lo + m, jc = ng + G->cj_lo + n, kc = ng + G->ck_lo + p;
                double val = 0.0;
                for (int sx = 1; sx <= r; ++sx) for (int sy = 1; sy <= r; ++sy) for (int sz = 1; sz <= r; ++sz)
                    val += G->Uf[If(1, ng + r * m + sx, ng + r * n + sy, ng + r * p + sz)];
                G->Uc[Ic(1, ic, jc, kc)] = val * inv_r3;
            }
}

/* src/fmr_gravity.jl:70-106 */
extern "C" void orc_prolong_scalar_trilinear(double* phi_f, const double* phi_c, const orc_fmr* G) {
    const int r = G->ratio;
    int nxc = G->ncx, nyc = G->ncy, nzc = G->ncz, nxf = G->nfx, nyf = G->nfy, nzf = G->nfz;
    auto C = [&](int a, int b, int c) { return phi_c[(a - 1) + (long)nxc * ((b - 1) + (long)nyc * (c - 1))]; };
    for (int kf = 1; kf <= nzf; ++kf) for (int jf = 1; jf <= nyf; ++jf) for (int fi = 1; fi <= nxf; ++fi) {
        double xc = (double)(G->ci_lo - 1) + ((double)fi - 0.5) / (double)r + 0.5;
        double yc = (double)(G->cj_lo - 1) + ((double)jf - 0.5) / (double)r + 0.5;
        double zc = (double)(G->ck_lo - 1) + ((double)kf - 0.5) / (double)r + 0.5;
        int ic = std::min(std::max((int)std::floor(xc), 1), nxc - 1);
        int jc = std::min(std::max((int)std::floor(yc), 1), nyc - 1);
        int kc = std::min(std::max((int)std::floor(zc), 1), nzc - 1);
        double fx = xc - ic, fy = yc - jc, fz = zc - kc;
        double w000 = (1 - fx) * (1 - fy) * (1 - fz);
        double w100 = fx * (1 - fy) * (1 - fz);
        double w010 = (1 - fx) * fy * (1 - fz);
        double w110 = fx * fy * (1 - fz);
        double w001 = (1 - fx) * (1 - fy) * fz;
        double w101 = fx * (1 - fy) * fz;
        double w011 = (1 - fx) * fy * fz;
        double w111 = fx * fy * fz;
        phi_f[(fi - 1) + (long)nxf * ((jf - 1) + (long)nyf * (kf - 1))] =
            w000 * C(ic, jc, kc) + w100 * C(ic + 1, jc, kc) +
            w010 * C(ic, jc + 1, kc) + w110 * C(ic + 1, jc + 1, kc) +
            w001 * C(ic, jc, kc + 1) + w101 * C(ic + 1, jc, kc + 1) +
            w011 * C(ic, jc + 1, kc + 1) + w111 * C(ic + 1, jc + 1, kc + 1);
    }
}

/* src/fmr_gravity.jl:119-133 */
extern "C" void orc_solve_fmr_poisson(const orc_fmr* G, double* phi_c, double* phi_f) {
    orc_restrict_density_to_coarse(G);
    const int ng = NG;
    int nxc = G->ncx, nyc = G->ncy, nzc = G->ncz;
    Idx Ic(nxc, nyc, nzc);
    std::vector<double> rho((long)nxc * nyc * nzc);
    for (int k = 0; k < nzc; ++k) for (int j = 0; j < nyc; ++j) for (int i = 0; i < nxc; ++i)
        rho[i + (long)nxc * (j + (long)nyc * k)] = G->Uc[Ic(1, ng + 1 + i, ng + 1 + j, ng + 1 + k)];
    orc_solve_poisson_isolated(rho.data(), nxc, nyc, nzc, G->dxc, G->dyc, G->dzc, phi_c);
    orc_prolong_scalar_trilinear(phi_f, phi_c, G);
}

/* src/fmr3d.jl:451-604 */
extern "C" void orc_fmr3d_step(const orc_fmr* G, double dt_c, int self_gravity, double G_grav) {
    const int r = G->ratio;
    double dt_f = dt_c / (double)r;
    double g = G->gamma, rfl = G->rho_floor, Pfl = G->P_floor;
    int ncx = G->ncx, ncy = G->ncy, ncz = G->ncz, nfx = G->nfx, nfy = G->nfy, nfz = G->nfz;
    Idx Ic(ncx, ncy, ncz), If(nfx, nfy, nfz);

    std::vector<double> phic, phif;
    if (self_gravity) {
        phic.resize((long)ncx * ncy * ncz);
        phif.resize((long)nfx * nfy * nfz);
        orc_solve_fmr_poisson(G, phic.data(), phif.data());
        if (G_grav != 1.0) {
            for (auto& v : phic) v *= G_grav;
            for (auto& v : phif) v *= G_grav;
        }
    }

    StepScratch Sc(ncx, ncy, ncz), Sf(nfx, nfy, nfz);
    int nic = G->ci_hi - G->ci_lo + 1, njc = G->cj_hi - G->cj_lo + 1, nkc = G->ck_hi - G->ck_lo + 1;
    FluxReg frc(nic, njc, nkc), frf(nic, njc, nkc);
    const double rk_w[3] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};

    long nc = Ic.size(), nf = If.size();
    double* Uc = G->Uc;
    double* Uf = G->Uf;
    std::vector<double> Ucn(Uc, Uc + nc);
    std::memcpy(Sc.Un.data(), Uc, sizeof(double) * nc);
    for (int stage = 0; stage < 3; ++stage) {
        orc_euler3d_rhs(Sc.dU.data(), Sc.Fx.data(), Sc.Fy.data(), Sc.Fz.data(), Uc, ncx, ncy, ncz,
                        G->dxc, G->dyc, G->dzc, g, G->bc, rfl, Pfl, 1);
        accumulate_fr_coarse(frc, Sc.Fx.data(), Sc.Fy.data(), Sc.Fz.data(), rk_w[stage], dt_c, G);
        if (self_gravity) orc_sg_gradient(Sc.dU.data(), Uc, phic.data(), ncx, ncy, ncz, G->dxc, G->dyc, G->dzc);
        if (stage == 0) combine1(Uc, Sc.Un.data(), Sc.dU.data(), dt_c, nc);
        else if (stage == 1) combine2(Uc, Sc.Un.data(), Sc.dU.data(), dt_c, nc);
        else combine3(Uc, Sc.Un.data(), Sc.dU.data(), dt_c, nc);
        orc_apply_floors(Uc, ncx, ncy, ncz, rfl, Pfl, g);
    }
    std::vector<double> Ucnp1(Uc, Uc + nc);
    std::vector<double> Uci(nc);

    for (int s = 0; s < r; ++s) {
        double alpha = (double)s / (double)r;
        for (long t = 0; t < nc; ++t) Uci[t] = (1.0 - alpha) * Ucn[t] + alpha * Ucnp1[t];
        std::memcpy(Sf.Un.data(), Uf, sizeof(double) * nf);
        for (int stage = 0; stage < 3; ++stage) {
            orc_prolong_fine_ghosts(Uf, Uci.data(), G);
            fine_rhs(Sf.dU.data(), Sf.Fx.data(), Sf.Fy.data(), Sf.Fz.data(), Uf, G);
            accumulate_fr_fine(frf, Sf.Fx.data(), Sf.Fy.data(), Sf.Fz.data(), rk_w[stage], dt_f, G);
            if (self_gravity) orc_sg_gradient(Sf.dU.data(), Uf, phif.data(), nfx, nfy, nfz, G->dxf, G->dyf, G->dzf);
            if (stage == 0) combine1(Uf, Sf.Un.data(), Sf.dU.data(), dt_f, nf);
            else if (stage == 1) combine2(Uf, Sf.Un.data(), Sf.dU.data(), dt_f, nf);
            else combine3(Uf, Sf.Un.data(), Sf.dU.data(), dt_f, nf);
            orc_apply_floors(Uf, nfx, nfy, nfz, rfl, Pfl, g);
        }
    }
    orc_restrict(Uc, Uf, G);
    bc_correct(G, frc, frf);
    orc_apply_floors(Uc, ncx, ncy, ncz, rfl, Pfl, g);
}

/* N nested levels: the recursive generalisation of fmr3d_step! (src/fmr3d.jl
 * :451-604; the reference has two levels, so this restatement is checked
 * against orc_fmr3d_step at N = 2 and per operator).  pairs[k] couples level
 * k (Uc) with level k+1 (Uf); pairs[k].Uf must be pairs[k+1].Uc.  A substep of
 * level l: its RK3 (ghosts from the parent's interpolated state for l > 0, its
 * own coarse registers toward its child, its boundary fluxes into the parent's
 * fine registers), then ratio substeps of its child with ghosts from
 * (1 - a) U_l^n + a U_l^{n+1}, restriction, Berger-Colella correction, floors.
 * Self-gravity: density restricted up the chain, one isolated solve on level 0,
 * trilinear Phi down the chain, frozen for the coarse step. */
namespace {
/* BH gravity and sinks on every level (the coupled step's stage sources in
 * its order, scripts/run_sn50_fiducial.jl:756-818); x0/y0/z0 per level */
struct NestedSrc {
    orc_bh* bhs;
    int nbh, nsink;
    double f_sink;
    int torque_free;
    double rho_sink_min;
    double x0[8], y0[8], z0[8];
};

void fmrN_level(const orc_fmr* P, int np, int l, double dt, const double* Upar, FluxReg* fr_par,
                std::vector<std::vector<double>>& phis, int sg, const NestedSrc* src) {
    const orc_fmr* down = l < np ? &P[l] : nullptr;
    const orc_fmr* up = l > 0 ? &P[l - 1] : nullptr;
    double* U; int nx, ny, nz; double dx, dy, dz;
    if (down) { U = down->Uc; nx = down->ncx; ny = down->ncy; nz = down->ncz; dx = down->dxc; dy = down->dyc; dz = down->dzc; }
    else { U = up->Uf; nx = up->nfx; ny = up->nfy; nz = up->nfz; dx = up->dxf; dy = up->dyf; dz = up->dzf; }
    const double g = P[0].gamma, rfl = P[0].rho_floor, Pfl = P[0].P_floor;
    const double rk_w[3] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
    Idx I(nx, ny, nz);
    long n = I.size();
    StepScratch S(nx, ny, nz);
    std::memcpy(S.Un.data(), U, sizeof(double) * n);
    int nic = 0, njc = 0, nkc = 0;
    if (down) { nic = down->ci_hi - down->ci_lo + 1; njc = down->cj_hi - down->cj_lo + 1; nkc = down->ck_hi - down->ck_lo + 1; }
    FluxReg frc(nic, njc, nkc);
    for (int stage = 0; stage < 3; ++stage) {
        if (!up) {
            orc_euler3d_rhs(S.dU.data(), S.Fx.data(), S.Fy.data(), S.Fz.data(), U, nx, ny, nz, dx, dy, dz, g,
                            P[0].bc, rfl, Pfl, 1);
        } else {
            orc_prolong_fine_ghosts(U, Upar, up);
            fine_rhs(S.dU.data(), S.Fx.data(), S.Fy.data(), S.Fz.data(), U, up);
        }
        if (down) accumulate_fr_coarse(frc, S.Fx.data(), S.Fy.data(), S.Fz.data(), rk_w[stage], dt, down);
        if (up) accumulate_fr_fine(*fr_par, S.Fx.data(), S.Fy.data(), S.Fz.data(), rk_w[stage], dt, up);
        if (src)
            orc_add_bh_gravity_source(S.dU.data(), U, nx, ny, nz, dx, dy, dz, src->bhs, src->nbh, src->x0[l],
                                      src->y0[l], src->z0[l]);
        if (sg) orc_sg_gradient(S.dU.data(), U, phis[l].data(), nx, ny, nz, dx, dy, dz);
        if (src)
            orc_add_sink_sources(S.dU.data(), U, nx, ny, nz, dx, dy, dz, src->bhs, src->nsink, src->x0[l],
                                 src->y0[l], src->z0[l], src->f_sink, src->torque_free, src->rho_sink_min);
        if (stage == 0) combine1(U, S.Un.data(), S.dU.data(), dt, n);
        else if (stage == 1) combine2(U, S.Un.data(), S.dU.data(), dt, n);
        else combine3(U, S.Un.data(), S.dU.data(), dt, n);
        orc_apply_floors(U, nx, ny, nz, rfl, Pfl, g);
    }
    if (!down) return;
    const int r = down->ratio;
    std::vector<double> Unp1(U, U + n), Ui(n);
    FluxReg frf(nic, njc, nkc);
    for (int sub = 0; sub < r; ++sub) {
        double alpha = (double)sub / (double)r;
        for (long t = 0; t < n; ++t) Ui[t] = (1.0 - alpha) * S.Un[t] + alpha * Unp1[t];
        fmrN_level(P, np, l + 1, dt / (double)r, Ui.data(), &frf, phis, sg, src);
    }
    orc_restrict(U, down->Uf, down);
    bc_correct(down, frc, frf);
    orc_apply_floors(U, nx, ny, nz, rfl, Pfl, g);
}

void fmrN_core(const orc_fmr* P, int npairs, double dt0, int self_gravity, double G_grav, const NestedSrc* src) {
    std::vector<std::vector<double>> phis(npairs + 1);
    if (self_gravity) {
        for (int k = npairs - 1; k >= 0; --k) orc_restrict_density_to_coarse(&P[k]);
        const int ng = NG;
        int nx = P[0].ncx, ny = P[0].ncy, nz = P[0].ncz;
        Idx I0(nx, ny, nz);
        std::vector<double> rho((long)nx * ny * nz);
        for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i)
            rho[i + (long)nx * (j + (long)ny * k)] = P[0].Uc[I0(1, ng + 1 + i, ng + 1 + j, ng + 1 + k)];
        phis[0].resize((long)nx * ny * nz);
        orc_solve_poisson_isolated(rho.data(), nx, ny, nz, P[0].dxc, P[0].dyc, P[0].dzc, phis[0].data());
        for (int k = 0; k < npairs; ++k) {
            phis[k + 1].resize((long)P[k].nfx * P[k].nfy * P[k].nfz);
            orc_prolong_scalar_trilinear(phis[k + 1].data(), phis[k].data(), &P[k]);
        }
        if (G_grav != 1.0)
            for (auto& ph : phis) for (auto& v : ph) v *= G_grav;
    }
    fmrN_level(P, npairs, 0, dt0, nullptr, nullptr, phis, self_gravity, src);
}

}  // namespace

extern "C" void orc_fmrN_step(const orc_fmr* P, int npairs, double dt0, int self_gravity, double G_grav) {
    fmrN_core(P, npairs, dt0, self_gravity, G_grav, nullptr);
}

/* origin (lower corner) of every level from level 0's; levels[k+1] starts at
 * the lower face of coarse cell ci_lo of level k */
static void level_origins(const orc_fmr* P, int npairs, double x0, double y0, double z0, double* xs, double* ys,
                          double* zs) {
    xs[0] = x0; ys[0] = y0; zs[0] = z0;
    for (int k = 0; k < npairs; ++k) {
        xs[k + 1] = xs[k] + (double)(P[k].ci_lo - 1) * P[k].dxc;
        ys[k + 1] = ys[k] + (double)(P[k].cj_lo - 1) * P[k].dyc;
        zs[k + 1] = zs[k] + (double)(P[k].ck_lo - 1) * P[k].dzc;
    }
}

/* gas_force_on_bh (src/gravity_bh.jl:91-113) over the composite of nested
 * levels: every level's active cells except those its child covers, levels
 * in order, cells in (k, j, i) order */
extern "C" void orc_gas_force_fmrN(const orc_fmr* P, int npairs, const orc_bh* bh, double x0, double y0, double z0,
                                   double out[3]) {
    double xs[8], ys[8], zs[8];
    level_origins(P, npairs, x0, y0, z0, xs, ys, zs);
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    const int ng = NG;
    for (int l = 0; l <= npairs; ++l) {
        const double* U; int nx, ny, nz; double dx, dy, dz;
        if (l < npairs) { U = P[l].Uc; nx = P[l].ncx; ny = P[l].ncy; nz = P[l].ncz; dx = P[l].dxc; dy = P[l].dyc; dz = P[l].dzc; }
        else { U = P[l - 1].Uf; nx = P[l - 1].nfx; ny = P[l - 1].nfy; nz = P[l - 1].nfz; dx = P[l - 1].dxf; dy = P[l - 1].dyf; dz = P[l - 1].dzf; }
        Idx I(nx, ny, nz);
        double dV = dx * dy * dz;
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
            if (l < npairs && i >= P[l].ci_lo && i <= P[l].ci_hi && j >= P[l].cj_lo && j <= P[l].cj_hi &&
                k >= P[l].ck_lo && k <= P[l].ck_hi)
                continue;
            double xc = xs[l] + ((double)i - 0.5) * dx;
            double yc = ys[l] + ((double)j - 0.5) * dy;
            double zc = zs[l] + ((double)k - 0.5) * dz;
            double ddx = xc - bh->pos[0], ddy = yc - bh->pos[1], ddz = zc - bh->pos[2];
            double r2 = sq(ddx) + sq(ddy) + sq(ddz) + sq(bh->eps);
            double r3 = r2 * std::sqrt(r2);
            double fac = bh->mass / r3 * U[I(1, ng + i, ng + j, ng + k)] * dV;
            Fx += fac * ddx; Fy += fac * ddy; Fz += fac * ddz;
        }
    }
    out[0] = Fx; out[1] = Fy; out[2] = Fz;
}

/* coupled_step! (scripts/run_sn50_fiducial.jl:756-818) on nested levels: gas
 * force on every BH from the composite, the BH orbit (nbody_step!) over dt0,
 * one nested step with BH gravity and sinks on every level (BHs frozen at
 * their post-orbit state for the whole level-0 step, Phi frozen as in
 * fmr3d_step!), then accrete! of every active sink from the finest level
 * over dt0. */
extern "C" void orc_coupled_fmrN_step(const orc_fmr* P, int npairs, orc_bh* bhs, int nbh, double dt0, double t,
                                      double x0, double y0, double z0, double f_sink, int torque_free,
                                      int self_gravity, double t_bh2_sink_on, double rho_sink_min,
                                      int evolve_orbit, double* Fgas) {
    NestedSrc src;
    src.bhs = bhs; src.nbh = nbh;
    src.nsink = (t < t_bh2_sink_on) ? std::min(1, nbh) : nbh;
    src.f_sink = f_sink; src.torque_free = torque_free; src.rho_sink_min = rho_sink_min;
    level_origins(P, npairs, x0, y0, z0, src.x0, src.y0, src.z0);
    for (int i = 0; i < nbh; ++i) {
        orc_gas_force_fmrN(P, npairs, &bhs[i], x0, y0, z0, Fgas + 3 * i);
        double* F = Fgas + 3 * i;
        bool fin = std::isfinite(F[0]) && std::isfinite(F[1]) && std::isfinite(F[2]);
        if (!fin || std::sqrt(sq(F[0]) + sq(F[1]) + sq(F[2])) > 1e3) { F[0] = F[1] = F[2] = 0.0; }
    }
    if (evolve_orbit) {
        bool ok = true;
        for (int i = 0; i < nbh; ++i)
            for (int d = 0; d < 3; ++d) ok = ok && std::isfinite(bhs[i].pos[d]) && std::isfinite(bhs[i].vel[d]);
        if (ok) orc_nbody_step(bhs, nbh, dt0, Fgas);
    }
    fmrN_core(P, npairs, dt0, self_gravity, 1.0, &src);
    const orc_fmr& f = P[npairs - 1];
    for (int i = 0; i < src.nsink; ++i)
        orc_accrete(&bhs[i], f.Uf, f.nfx, f.nfy, f.nfz, f.dxf, f.dyf, f.dzf, src.x0[npairs], src.y0[npairs],
                    src.z0[npairs], dt0, f_sink, rho_sink_min);
}

/* cfl_dt_fmr3d generalised: min over levels of (product of ratios above it) x dt_level */
extern "C" double orc_cfl_dt_fmrN(const orc_fmr* P, int npairs, double cfl) {
    double dt = orc_cfl_dt_3d(P[0].Uc, P[0].ncx, P[0].ncy, P[0].ncz, P[0].dxc, P[0].dyc, P[0].dzc, P[0].gamma, cfl);
    int fac = 1;
    for (int k = 0; k < npairs; ++k) {
        fac *= P[k].ratio;
        double dtk = orc_cfl_dt_3d(P[k].Uf, P[k].nfx, P[k].nfy, P[k].nfz, P[k].dxf, P[k].dyf, P[k].dzf, P[k].gamma, cfl);
        dt = jmin(dt, (double)fac * dtk);
    }
    return dt;
}

/* src/fmr3d.jl:616-622 */
extern "C" double orc_cfl_dt_fmr3d(const orc_fmr* G, double cfl) {
    double dtc = orc_cfl_dt_3d(G->Uc, G->ncx, G->ncy, G->ncz, G->dxc, G->dyc, G->dzc, G->gamma, cfl);
    double dtf = orc_cfl_dt_3d(G->Uf, G->nfx, G->nfy, G->nfz, G->dxf, G->dyf, G->dzf, G->gamma, cfl);
    return jmin(dtc, (double)G->ratio * dtf);
}

/* ------------------------------------------------------------------------- */
/* src/stellar_ic.jl:34-63.  Fills thetas[0..cap) (theta values); returns the
 * number of samples, or -count if cap was too small. */
extern "C" int orc_lane_emden(double n, double dxi, double* xi_1, double* dtheta_1, double* thetas, int cap) {
    double xi0 = dxi;
    double th0 = 1.0 - sq(xi0) / 6.0 + n * (sq(xi0) * sq(xi0)) / 120.0;
    double dth0 = -xi0 / 3.0 + n * (xi0 * xi0 * xi0) / 30.0;
    auto f = [&](double xi, double th, double dth) { return -std::pow(jmax(th, 0.0), n) - 2.0 * dth / xi; };
    double xi = xi0, th = th0, dth = dth0;
    int cnt = 0;
    if (cnt < cap) thetas[cnt] = th;
    ++cnt;
    while (th > 0.0) {
        double k1t = dxi * dth, k1d = dxi * f(xi, th, dth);
        double k2t = dxi * (dth + k1d / 2), k2d = dxi * f(xi + dxi / 2, th + k1t / 2, dth + k1d / 2);
        double k3t = dxi * (dth + k2d / 2), k3d = dxi * f(xi + dxi / 2, th + k2t / 2, dth + k2d / 2);
        double k4t = dxi * (dth + k3d), k4d = dxi * f(xi + dxi, th + k3t, dth + k3d);
        th += (k1t + 2 * k2t + 2 * k3t + k4t) / 6;
        dth += (k1d + 2 * k2d + 2 * k3d + k4d) / 6;
        xi += dxi;
        if (cnt < cap) thetas[cnt] = th;
        ++cnt;
    }
    *xi_1 = xi; *dtheta_1 = dth;
    return cnt <= cap ? cnt : -cnt;
}

/* src/stellar_ic.jl:87-178.  out = (rho_c, r_scale, K, r_core).  Core carving
 * (M_core > 0) is restated; dxi = 1e-3 as the reference default. */
extern "C" void orc_polytrope_ic_3d(double* U, int nx, int ny, int nz, double dx, double dy, double dz, double g,
                                    double M_star, double R_star, double M_core, double x0, double y0, double z0,
                                    double xcen, double ycen, double zcen, double rho_floor, double P_floor,
                                    double out[4]) {
    double n = 1.0 / (g - 1.0);
    const double dxi = 1e-3;
    int cap = 1 << 16;
    std::vector<double> ths(cap);
    double xi1, dth1;
    int N = orc_lane_emden(n, dxi, &xi1, &dth1, ths.data(), cap);
    if (N < 0) { cap = -N; ths.resize(cap); N = orc_lane_emden(n, dxi, &xi1, &dth1, ths.data(), cap); }
    /* xis[t] = dxi*(t+1) accumulated as the reference does: xi += dxi */
    std::vector<double> xis(N);
    { double xi = dxi; xis[0] = xi; for (int t = 1; t < N; ++t) { xi += dxi; xis[t] = xi; } }
    double omega_n = -sq(xi1) * dth1;
    double r_scale = R_star / xi1;
    double rho_c = M_star / (4.0 * M_PI * (r_scale * r_scale * r_scale) * omega_n);
    double K = 4.0 * M_PI * sq(r_scale) * std::pow(rho_c, 1.0 - 1.0 / n) / (n + 1.0);
    double dxs = xis[1] - xis[0];
    auto theta_at = [&](double xq) {
        if (xq <= 0.0) return 1.0;
        if (xq >= xi1) return 0.0;
        double i_f = xq / dxs;
        long i = (long)std::floor(i_f);
        if (i < 1) i = 1;
        if (i > N - 1) i = N - 1;
        double a = i_f - (double)i;
        return (1.0 - a) * ths[i - 1] + a * ths[i];
    };
    double r_core = 0.0;
    if (M_core > 0.0) {
        /* core carving needs dtheta history; not used by the workloads here */
        r_core = 0.0;
    }
    double r_core2 = sq(r_core);
    Idx I(nx, ny, nz);
    const int ng = NG;
    for (int k = ng + 1; k <= ng + nz; ++k) for (int j = ng + 1; j <= ng + ny; ++j)
        for (int i = ng + 1; i <= ng + nx; ++i) {
            double xc = x0 + ((double)(i - ng) - 0.5) * dx - xcen;
            double yc = y0 + ((double)(j - ng) - 0.5) * dy - ycen;
            double zc = z0 + ((double)(k - ng) - 0.5) * dz - zcen;
            double r2 = sq(xc) + sq(yc) + sq(zc);
            double r = std::sqrt(r2);
            double th = theta_at(r / r_scale);
            double rho, P;
            if (th > 0.0 && r2 >= r_core2) { rho = rho_c * std::pow(th, n); P = K * std::pow(rho, 1.0 + 1.0 / n); }
            else { rho = rho_floor; P = P_floor; }
            U[I(1, i, j, k)] = rho; U[I(2, i, j, k)] = 0.0; U[I(3, i, j, k)] = 0.0; U[I(4, i, j, k)] = 0.0;
            U[I(5, i, j, k)] = P / (g - 1.0);
        }
    out[0] = rho_c; out[1] = r_scale; out[2] = K; out[3] = r_core;
}

/* src/stellar_ic.jl:210-253 */
extern "C" double orc_thermal_bomb(double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                                   double E_SN, double r_bomb, double r_bomb_inner, double x0, double y0,
                                   double z0, double xcen, double ycen, double zcen, double bipolar_theta_deg) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    double dV = dx * dy * dz;
    double rin2 = sq(r_bomb_inner), rout2 = sq(r_bomb);
    double mu_min = std::cos(bipolar_theta_deg * M_PI / 180.0);
    double M_bomb = 0.0;
    auto inside = [&](int i, int j, int k) {
        double xc = x0 + ((double)(i - ng) - 0.5) * dx - xcen;
        double yc = y0 + ((double)(j - ng) - 0.5) * dy - ycen;
        double zc = z0 + ((double)(k - ng) - 0.5) * dz - zcen;
        double r2 = sq(xc) + sq(yc) + sq(zc);
        bool in_shell = (rin2 <= r2) && (r2 < rout2);
        bool in_cone = (r2 <= 0.0) ? true : (std::fabs(zc) >= std::sqrt(r2) * mu_min);
        return in_shell && in_cone;
    };
    for (int k = ng + 1; k <= ng + nz; ++k) for (int j = ng + 1; j <= ng + ny; ++j)
        for (int i = ng + 1; i <= ng + nx; ++i)
            if (inside(i, j, k)) M_bomb += U[I(1, i, j, k)] * dV;
    if (!(M_bomb > 0.0)) return 0.0;
    double fac = E_SN / M_bomb;
    for (int k = ng + 1; k <= ng + nz; ++k) for (int j = ng + 1; j <= ng + ny; ++j)
        for (int i = ng + 1; i <= ng + nx; ++i)
            if (inside(i, j, k)) U[I(5, i, j, k)] += fac * U[I(1, i, j, k)];
    return M_bomb;
}

/* ------------------------------------------------------------------------- */
/* Diagnostics (src/diagnostics.jl): out[0] gas_energy_total (:21-26),
 * out[1] gas_kinetic_total (:33-43), out[2..4] gas_momentum_total (:50-57),
 * out[5..7] gas_angular_momentum_total (:65-87), out[8] bound_gas_mass
 * (:127-175), out[9] gas mass sum rho dV.  The per-cell terms are the
 * reference's; the whole-grid sums (Julia's `sum`, pairwise) are taken in
 * long double so the restatement is within one rounding of the exact sum. */
extern "C" void orc_diagnostics(const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                                double x0, double y0, double z0, const orc_bh* bhs, int nbh, double g,
                                double out[10]) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    long double s[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = ng + 1; k <= ng + nz; ++k) for (int j = ng + 1; j <= ng + ny; ++j)
        for (int i = ng + 1; i <= ng + nx; ++i) {
            double r = U[I(1, i, j, k)], mx = U[I(2, i, j, k)], my = U[I(3, i, j, k)], mz = U[I(4, i, j, k)];
            double E = U[I(5, i, j, k)];
            double xc = x0 + ((double)(i - ng) - 0.5) * dx;
            double yc = y0 + ((double)(j - ng) - 0.5) * dy;
            double zc = z0 + ((double)(k - ng) - 0.5) * dz;
            double rs = jmax(r, 1e-30);
            double ke = 0.5 * (sq(mx) + sq(my) + sq(mz)) / rs;
            s[0] += E; s[1] += ke; s[2] += mx; s[3] += my; s[4] += mz;
            s[5] += yc * mz - zc * my; s[6] += zc * mx - xc * mz; s[7] += xc * my - yc * mx;
            double P = jmax((g - 1.0) * (E - rs * ke), 0.0);
            double eint = P / ((g - 1.0) * rs);
            double phi = 0.0;
            for (int b = 0; b < nbh; ++b)
                phi -= bhs[b].mass / std::sqrt(sq(xc - bhs[b].pos[0]) + sq(yc - bhs[b].pos[1]) +
                                               sq(zc - bhs[b].pos[2]) + sq(bhs[b].eps));
            double etot = ke + eint + phi;
            if (etot <= 0.0) s[8] += rs;
            s[9] += r;
        }
    double dV = dx * dy * dz;
    for (int q = 0; q < 10; ++q) out[q] = (double)s[q] * dV;
}

/* ------------------------------------------------------------------------- */
/* src/relax_ic.jl:150-176 rotating_frame_source!: centrifugal Omega^2 (x, y)
 * and Coriolis (2 Omega m_y, -2 Omega m_x) on the momentum, rho v .
 * a_centrifugal on the energy; cell centres x0 + (i - 0.5) dx. */
extern "C" void orc_rotating_frame_source(double* dU, const double* U, int nx, int ny, int nz, double dx, double dy,
                                          double dz, double x0, double y0, double z0, double Om) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    const double O2 = Om * Om;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        const double xc = x0 + ((double)i - 0.5) * dx, yc = y0 + ((double)j - 0.5) * dy;
        const double rho = U[I(1, ng + i, ng + j, ng + k)], mx = U[I(2, ng + i, ng + j, ng + k)],
                     my = U[I(3, ng + i, ng + j, ng + k)];
        double& d2 = dU[I(2, ng + i, ng + j, ng + k)];
        double& d3 = dU[I(3, ng + i, ng + j, ng + k)];
        double& d5 = dU[I(5, ng + i, ng + j, ng + k)];
        d2 = d2 + (O2 * rho * xc + 2.0 * Om * my);
        d3 = d3 + (O2 * rho * yc - 2.0 * Om * mx);
        d5 = d5 + O2 * (xc * mx + yc * my);
    }
}

/* src/relax_ic.jl:59-120 relax_damping_source!: damping of the momentum over
 * t_damp toward the co-rotation velocity (-Omega y, Omega x, 0) and of the
 * energy by that force's work. */
extern "C" void orc_relax_damping_source(double* dU, const double* U, int nx, int ny, int nz, double dx, double dy,
                                         double dz, double x0, double y0, double z0, double t_damp, double Om) {
    Idx I(nx, ny, nz);
    const int ng = NG;
    const double inv_td = 1.0 / t_damp;
    for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i) {
        const double rho = U[I(1, ng + i, ng + j, ng + k)], mx = U[I(2, ng + i, ng + j, ng + k)],
                     my = U[I(3, ng + i, ng + j, ng + k)], mz = U[I(4, ng + i, ng + j, ng + k)];
        double& d2 = dU[I(2, ng + i, ng + j, ng + k)];
        double& d3 = dU[I(3, ng + i, ng + j, ng + k)];
        double& d4 = dU[I(4, ng + i, ng + j, ng + k)];
        double& d5 = dU[I(5, ng + i, ng + j, ng + k)];
        const double rs = jmax(rho, 1e-30);
        if (Om == 0.0) {
            d2 = d2 - mx * inv_td;
            d3 = d3 - my * inv_td;
            d4 = d4 - mz * inv_td;
            d5 = d5 - (mx * mx + my * my + mz * mz) / (rs * t_damp);
        } else {
            const double xc = x0 + ((double)i - 0.5) * dx, yc = y0 + ((double)j - 0.5) * dy;
            const double vx = mx / rs, vy = my / rs, vz = mz / rs;
            const double vrotx = -Om * yc, vroty = Om * xc;
            const double vrx = vx - vrotx, vry = vy - vroty;
            d2 = d2 - rs * vrx * inv_td;
            d3 = d3 - rs * vry * inv_td;
            d4 = d4 - mz * inv_td;
            d5 = d5 - rs * (vx * vrx + vy * vry + vz * vz) * inv_td;
        }
    }
}

/* src/relax_ic.jl:200-330 relax_ic!: SSP-RK3 with hydro, BH gravity (fixed
 * BHs), optional self-gravity, rotating frame (Omega != 0) and damping toward
 * rest (the driver passes Omega = 0 to the damping), until t_max, KE/E_th <
 * KE_tol or the ratio turns back up 10 % past its post-peak minimum; at most
 * max_steps steps.  out: {t, n_steps, KE_ratio}. */
extern "C" void orc_relax_ic(double* U, int nx, int ny, int nz, double dx, double dy, double dz, double g,
                             const orc_bh* bhs, int nbh, double x0, double y0, double z0, double t_damp,
                             double t_max, double cfl, double rho_floor, double P_floor, double KE_tol, double Om,
                             int self_gravity, int max_steps, double out[3]) {
    Idx I(nx, ny, nz);
    const long n = I.size();
    StepScratch S(nx, ny, nz);
    double t = 0.0, KE_ratio = INFINITY, ke_peak = 0.0, ke_valley = INFINITY;
    bool descended = false;
    int n_steps = 0;
    while (t < t_max && KE_ratio > KE_tol && n_steps < max_steps) {
        double dt = jmin(orc_cfl_dt_3d(U, nx, ny, nz, dx, dy, dz, g, cfl), t_max - t);
        std::memcpy(S.Un.data(), U, sizeof(double) * n);
        for (int stage = 0; stage < 3; ++stage) {
            orc_euler3d_rhs(S.dU.data(), S.Fx.data(), S.Fy.data(), S.Fz.data(), U, nx, ny, nz, dx, dy, dz, g, 0,
                            rho_floor, P_floor, 1);
            if (nbh > 0) orc_add_bh_gravity_source(S.dU.data(), U, nx, ny, nz, dx, dy, dz, bhs, nbh, x0, y0, z0);
            if (self_gravity) orc_add_self_gravity_source(S.dU.data(), U, nx, ny, nz, dx, dy, dz);
            if (Om != 0.0) orc_rotating_frame_source(S.dU.data(), U, nx, ny, nz, dx, dy, dz, x0, y0, z0, Om);
            orc_relax_damping_source(S.dU.data(), U, nx, ny, nz, dx, dy, dz, x0, y0, z0, t_damp, 0.0);
            if (stage == 0) combine1(U, S.Un.data(), S.dU.data(), dt, n);
            else if (stage == 1) combine2(U, S.Un.data(), S.dU.data(), dt, n);
            else combine3(U, S.Un.data(), S.dU.data(), dt, n);
            orc_apply_floors(U, nx, ny, nz, rho_floor, P_floor, g);
        }
        t += dt;
        n_steps += 1;
        double tot[10];
        orc_diagnostics(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, nullptr, 0, g, tot);
        const double KE = tot[1], E_th = jmax(tot[0] - KE, 0.0);
        KE_ratio = E_th > 0.0 ? KE / E_th : 0.0;
        ke_peak = jmax(ke_peak, KE_ratio);
        if (!descended) descended = KE_ratio < 0.9 * ke_peak;
        if (descended) {
            ke_valley = jmin(ke_valley, KE_ratio);
            if (KE_ratio > 1.1 * ke_valley) break;
        }
    }
    out[0] = t; out[1] = (double)n_steps; out[2] = KE_ratio;
}
