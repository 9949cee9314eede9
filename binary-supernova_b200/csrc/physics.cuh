// physics.cuh -- WENO5-Z, cell pressure, face energy and HLLC for the FP64
// path.  Every expression keeps the reference's evaluation order
// (a+b+c == (a+b)+c, a*b*c == (a*b)*c, x^2 == x*x) and this translation unit
// family is compiled with -fmad=false, IEEE division and square root, so the
// results are bit-identical to the reference's CPU path.
#pragma once

#include "bsn_internal.cuh"

namespace bsn {
namespace f64 {

// WENO-Z nonlinear weights and the weighted sum (src/weno5.jl:14-21, 40, 60).
__device__ __forceinline__ double wenoz_sum(double b0, double b1, double b2, double d0, double d1, double d2,
                                            double q0, double q1, double q2) {
    const double eps = 1e-36;
    double tau5 = fabs(b0 - b2);
    double a0 = d0 * (1.0 + sq(tau5 / (eps + b0)));
    double a1 = d1 * (1.0 + sq(tau5 / (eps + b1)));
    double a2 = d2 * (1.0 + sq(tau5 / (eps + b2)));
    double asum = a0 + a1 + a2;
    double w0 = a0 / asum, w1 = a1 / asum, w2 = a2 / asum;
    return w0 * q0 + w1 * q1 + w2 * q2;
}

// Left- and right-biased WENO5-Z values at the interface between c2 and c3
// from the six cells c0..c5 (src/weno5.jl:25-61).  The right reconstruction's
// first two candidate polynomials and its first smoothness indicator are the
// same expressions on the same cells as the left's q1, q2 and beta1, and the
// 13/12 term of left beta2 equals that of right beta1, so they are computed
// once; the values are unchanged bit for bit.
__device__ __forceinline__ void weno5_lr(double c0, double c1, double c2, double c3, double c4, double c5,
                                         double* L, double* R) {
    const double t13 = 1.0 / 3.0, m76 = -7.0 / 6.0, e116 = 11.0 / 6.0, m16 = -1.0 / 6.0, f56 = 5.0 / 6.0;
    const double k1312 = 13.0 / 12.0, k14 = 1.0 / 4.0;
    double qA = t13 * c0 + m76 * c1 + e116 * c2;   // left q0
    double qB = m16 * c1 + f56 * c2 + t13 * c3;    // left q1 == right q0
    double qC = t13 * c2 + f56 * c3 + m16 * c4;    // left q2 == right q1
    double qD = e116 * c3 + m76 * c4 + t13 * c5;   // right q2
    double bA = k1312 * sq(c0 - 2.0 * c1 + c2) + k14 * sq(c0 - 4.0 * c1 + 3.0 * c2);   // left b0
    double bB = k1312 * sq(c1 - 2.0 * c2 + c3) + k14 * sq(c1 - c3);                    // left b1 == right b0
    double s2 = k1312 * sq(c2 - 2.0 * c3 + c4);
    double bC = s2 + k14 * sq(3.0 * c2 - 4.0 * c3 + c4);                              // left b2
    double bD = s2 + k14 * sq(c2 - 4.0 * c3 + 3.0 * c4);                              // right b1
    double bE = k1312 * sq(c3 - 2.0 * c4 + c5) + k14 * sq(3.0 * c3 - 4.0 * c4 + c5);   // right b2
    *L = wenoz_sum(bA, bB, bC, 1.0 / 10.0, 6.0 / 10.0, 3.0 / 10.0, qA, qB, qC);
    *R = wenoz_sum(bB, bD, bE, 3.0 / 10.0, 6.0 / 10.0, 1.0 / 10.0, qB, qC, qD);
}

// src/euler3d.jl:86-90
__device__ __forceinline__ double cell_pressure(double r, double mx, double my, double mz, double E,
                                                double gm1) {
    r = jmax(r, 1e-30);
    double KE = 0.5 * (sq(mx) + sq(my) + sq(mz)) / r;
    return jmax(gm1 * (E - KE), 0.0);
}

// src/euler3d.jl:99-106
__device__ __forceinline__ double EL_from_P(double PL, double rL, double mxL, double myL, double mzL,
                                            double gm1) {
    double rp = jmax(rL, 1e-30);
    double m2 = sq(mxL) + sq(myL) + sq(mzL);
    double KE_raw = 0.5 * m2 / rp;
    double KE = jmin(KE_raw, 0.5 * rp * 1e4);
    return PL / gm1 + KE;
}

// HLLC along the normal (src/hllc.jl:17-165).  Inputs/outputs are in the
// rotated (normal, t1, t2) ordering.
__device__ __forceinline__ void hllc_normal(double rL, double mnL, double mt1L, double mt2L, double EL,
                                            double rR, double mnR, double mt1R, double mt2R, double ER,
                                            double g, double gm1, double F[5]) {
    if (rL <= 0.0) { rL = 1e-30; mnL = 0.0; mt1L = 0.0; mt2L = 0.0; EL = 0.0; }
    else           { rL = jmax(rL, 1e-30); }
    if (rR <= 0.0) { rR = 1e-30; mnR = 0.0; mt1R = 0.0; mt2R = 0.0; ER = 0.0; }
    else           { rR = jmax(rR, 1e-30); }

    double m2L = sq(mnL) + sq(mt1L) + sq(mt2L);
    if (m2L > sq(rL) * 1e4) {
        double s = rL * 100.0 / sqrt(m2L);
        mnL *= s; mt1L *= s; mt2L *= s;
    }
    double m2R = sq(mnR) + sq(mt1R) + sq(mt2R);
    if (m2R > sq(rR) * 1e4) {
        double s = rR * 100.0 / sqrt(m2R);
        mnR *= s; mt1R *= s; mt2R *= s;
    }
    double KE_L = jmin(0.5 * (sq(mnL) + sq(mt1L) + sq(mt2L)) / rL, 0.5 * rL * 1e4);
    double KE_R = jmin(0.5 * (sq(mnR) + sq(mt1R) + sq(mt2R)) / rR, 0.5 * rR * 1e4);
    EL = jmax(EL, KE_L);
    ER = jmax(ER, KE_R);

    double vnL = mnL / rL, vt1L = mt1L / rL, vt2L = mt2L / rL;
    double vnR = mnR / rR, vt1R = mt1R / rR, vt2R = mt2R / rR;
    double pL = gm1 * (EL - KE_L);
    double pR = gm1 * (ER - KE_R);
    double csL = sqrt(g * pL / rL);
    double csR = sqrt(g * pR / rR);

    double SL, SR;
    if (pL > 0.0 && pR > 0.0) {
        double r_avg = 0.5 * (rL + rR);
        double cs_avg = 0.5 * (csL + csR);
        double p_star = jmax(0.0, 0.5 * (pL + pR) - 0.5 * (vnR - vnL) * r_avg * cs_avg);
        double gg = (g + 1.0) / (2.0 * g);
        double qL = p_star > pL ? sqrt(1.0 + gg * (p_star / pL - 1.0)) : 1.0;
        double qR = p_star > pR ? sqrt(1.0 + gg * (p_star / pR - 1.0)) : 1.0;
        SL = vnL - csL * qL;
        SR = vnR + csR * qR;
    } else {
        SL = jmin(vnL - csL, vnR - csR);
        SR = jmax(vnL + csL, vnR + csR);
    }

    double denom = rL * (SL - vnL) - rR * (SR - vnR);
    if (fabs(denom) < 1e-100) { F[0] = F[1] = F[2] = F[3] = F[4] = 0.0; return; }
    double S_star = (pR - pL + rL * vnL * (SL - vnL) - rR * vnR * (SR - vnR)) / denom;

    double FrL = mnL, FmnL = rL * sq(vnL) + pL, Fmt1L = mt1L * vnL, Fmt2L = mt2L * vnL;
    double FEL = (EL + pL) * vnL;
    if (SL >= 0.0) { F[0] = FrL; F[1] = FmnL; F[2] = Fmt1L; F[3] = Fmt2L; F[4] = FEL; return; }
    double FrR = mnR, FmnR = rR * sq(vnR) + pR, Fmt1R = mt1R * vnR, Fmt2R = mt2R * vnR;
    double FER = (ER + pR) * vnR;
    if (SR <= 0.0) { F[0] = FrR; F[1] = FmnR; F[2] = Fmt1R; F[3] = Fmt2R; F[4] = FER; return; }

    if (jmax(rL, rR) > 3.0 * jmin(rL, rR)) {
        double inv_dS = 1.0 / (SR - SL);
        double SLSR = SL * SR;
        F[0] = (SR * FrL - SL * FrR + SLSR * (rR - rL)) * inv_dS;
        F[1] = (SR * FmnL - SL * FmnR + SLSR * (mnR - mnL)) * inv_dS;
        F[2] = (SR * Fmt1L - SL * Fmt1R + SLSR * (mt1R - mt1L)) * inv_dS;
        F[3] = (SR * Fmt2L - SL * Fmt2R + SLSR * (mt2R - mt2L)) * inv_dS;
        F[4] = (SR * FEL - SL * FER + SLSR * (ER - EL)) * inv_dS;
        return;
    }
    if (S_star >= 0.0) {
        double dL = rL * (SL - vnL);
        double chi = dL / (SL - S_star);
        double EsL = fabs(dL) > 1e-100 ? chi * (EL / rL + (S_star - vnL) * (S_star + pL / dL)) : 0.0;
        F[0] = FrL + SL * (chi - rL);
        F[1] = FmnL + SL * (chi * S_star - mnL);
        F[2] = Fmt1L + SL * (chi * vt1L - mt1L);
        F[3] = Fmt2L + SL * (chi * vt2L - mt2L);
        F[4] = FEL + SL * (EsL - EL);
    } else {
        double dR = rR * (SR - vnR);
        double chi = dR / (SR - S_star);
        double EsR = fabs(dR) > 1e-100 ? chi * (ER / rR + (S_star - vnR) * (S_star + pR / dR)) : 0.0;
        F[0] = FrR + SR * (chi - rR);
        F[1] = FmnR + SR * (chi * S_star - mnR);
        F[2] = Fmt1R + SR * (chi * vt1R - mt1R);
        F[3] = Fmt2R + SR * (chi * vt2R - mt2R);
        F[4] = FER + SR * (EsR - ER);
    }
}

// One interface along direction d from six cells (rows of 5 conserved
// values plus the cell pressure): WENO of rho, m, P (clamped to [0, stencil
// max]), energy from P, rotated HLLC (src/gpu_kernels.jl:51-154,
// src/hllc.jl:176-208).  F is returned in (rho, mx, my, mz, E) order.
template <int D>
__device__ __forceinline__ void interface_flux(const double (&c)[6][6], double g, double gm1, double F[5]) {
    double L[5], R[5];
#pragma unroll
    for (int q = 0; q < 4; ++q) weno5_lr(c[0][q], c[1][q], c[2][q], c[3][q], c[4][q], c[5][q], &L[q], &R[q]);
    double PL, PR;
    weno5_lr(c[0][5], c[1][5], c[2][5], c[3][5], c[4][5], c[5][5], &PL, &PR);
    double PmaxL = jmax(jmax(jmax(jmax(c[0][5], c[1][5]), c[2][5]), c[3][5]), c[4][5]);
    double PmaxR = jmax(jmax(jmax(jmax(c[1][5], c[2][5]), c[3][5]), c[4][5]), c[5][5]);
    PL = jclamp(PL, 0.0, PmaxL);
    PR = jclamp(PR, 0.0, PmaxR);
    double EL = EL_from_P(PL, L[0], L[1], L[2], L[3], gm1);
    double ER = EL_from_P(PR, R[0], R[1], R[2], R[3], gm1);
    double Fr[5];
    if (D == 0) {
        hllc_normal(L[0], L[1], L[2], L[3], EL, R[0], R[1], R[2], R[3], ER, g, gm1, Fr);
        F[0] = Fr[0]; F[1] = Fr[1]; F[2] = Fr[2]; F[3] = Fr[3]; F[4] = Fr[4];
    } else if (D == 1) {
        hllc_normal(L[0], L[2], L[1], L[3], EL, R[0], R[2], R[1], R[3], ER, g, gm1, Fr);
        F[0] = Fr[0]; F[1] = Fr[2]; F[2] = Fr[1]; F[3] = Fr[3]; F[4] = Fr[4];
    } else {
        hllc_normal(L[0], L[3], L[1], L[2], EL, R[0], R[3], R[1], R[2], ER, g, gm1, Fr);
        F[0] = Fr[0]; F[1] = Fr[2]; F[2] = Fr[3]; F[3] = Fr[1]; F[4] = Fr[4];
    }
}

// Density/pressure floors (src/gpu_kernels.jl:26-46).  Pfl_gm1 = P_floor/(gamma-1).
__device__ __forceinline__ void apply_floor(double& r, double& mx, double& my, double& mz, double& E,
                                            double rho_floor, double P_floor, double Pfl_gm1, double gm1) {
    if (r < rho_floor) {
        r = rho_floor; mx = 0.0; my = 0.0; mz = 0.0; E = Pfl_gm1;
    } else {
        double KE = 0.5 * (sq(mx) + sq(my) + sq(mz)) / r;
        double P = gm1 * (E - KE);
        if (P < P_floor) E = Pfl_gm1 + KE;
    }
}

// rotating_frame_source! (src/relax_ic.jl:150-176) on one cell's RHS d[5]:
// centrifugal rho Omega^2 (x, y) plus Coriolis 2 Omega (m_y, -m_x) on the
// momentum, rho v . a_centrifugal on the energy, in the reference's
// expression order.
__device__ __forceinline__ void rot_frame_src(double* d, double u0, double u1, double u2, double xc, double yc,
                                              double om) {
    const double O2 = om * om;
    d[1] = d[1] + (O2 * u0 * xc + 2.0 * om * u2);
    d[2] = d[2] + (O2 * u0 * yc - 2.0 * om * u1);
    d[4] = d[4] + O2 * (xc * u1 + yc * u2);
}

// relax_damping_source! (src/relax_ic.jl:59-120) on one cell's RHS d[5]:
// momentum damped toward the co-rotation velocity (-Omega y, Omega x, 0) over
// t_damp, the energy by the work of that force (inv_td = 1 / t_damp).
__device__ __forceinline__ void damp_src(double* d, double u0, double u1, double u2, double u3, double xc, double yc,
                                         double inv_td, double t_damp, double om) {
    const double rs = jmax(u0, 1e-30);
    if (om == 0.0) {
        d[1] = d[1] - u1 * inv_td;
        d[2] = d[2] - u2 * inv_td;
        d[3] = d[3] - u3 * inv_td;
        d[4] = d[4] - (u1 * u1 + u2 * u2 + u3 * u3) / (rs * t_damp);
    } else {
        const double vx = u1 / rs, vy = u2 / rs, vz = u3 / rs;
        const double vrotx = -om * yc, vroty = om * xc;
        const double vrx = vx - vrotx, vry = vy - vroty;
        d[1] = d[1] - rs * vrx * inv_td;
        d[2] = d[2] - rs * vry * inv_td;
        d[3] = d[3] - u3 * inv_td;
        d[4] = d[4] - rs * (vx * vrx + vy * vry + vz * vz) * inv_td;
    }
}

// CFL speed of one cell (src/gpu_kernels.jl:174-191).
__device__ __forceinline__ double cfl_speed(double U0, double U1, double U2, double U3, double U4, double g,
                                            double gm1, double idx, double idy, double idz) {
    double r = jmax(U0, 1e-30);
    double vx = U1 / r, vy = U2 / r, vz = U3 / r;
    double KE = 0.5 * (sq(vx) + sq(vy) + sq(vz));
    double P = jmax(gm1 * (U4 / r - KE) * r, 0.0);
    double cs = sqrt(g * P / r);
    return jmax(jmax((fabs(vx) + cs) * idx, (fabs(vy) + cs) * idy), (fabs(vz) + cs) * idz);
}

}  // namespace f64
}  // namespace bsn
