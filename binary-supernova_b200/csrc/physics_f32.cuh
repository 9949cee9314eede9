// physics_f32.cuh -- FP32 stencil physics of the fast path.
//
// Same method as the reference (WENO5-Z of rho, m, P with the P clamp, face
// energy from P, HLLC with its guards), evaluated in FP32 with approximate
// reciprocals/square roots (the translation units are built with --ftz=true
// --prec-div=false --prec-sqrt=false).  Every fused multiply-add is written
// out (fmaf, fma.rn.f32x2) and the units are built with --fmad=false, so no
// result depends on the compiler's contraction choices: each tile variant,
// and TMA or plain staging, gives the same bits.  FP32-specific guards:
//   * WENO-Z: tau/(eps+beta) is clamped to 1e18 before squaring, so the
//     weights cannot overflow to Inf/Inf when beta ~ 0 and tau != 0 (with the
//     reference's eps = 1e-36 the unclamped square overflows FP32);
//   * the 1e-100 guards of HLLC become 1e-36 (1e-100 is zero in FP32).
// Results differ from the FP64 path by rounding; their effect on the solution
// is reported as L1 errors against the FP64 oracle.
#pragma once

#include "bsn_internal.cuh"
#include "physics.cuh"

namespace bsn {
namespace f32 {

// Fast division (reciprocal approximation times the numerator).  Used where
// the denominator lies in [1e-36, 2^126): the WENO-Z denominators eps + beta
// and weight sums, densities floored at 1e-30, pressures, HLLC wave-speed
// differences; a denominator above 2^126 would need state values beyond
// 1e18, far outside what the path represents.
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

__device__ __forceinline__ float wz(float b0, float b1, float b2, float d0, float d1, float d2, float q0, float q1,
                                    float q2) {
    const float eps = 1e-36f, cap = 1e18f;
    float tau = fabsf(b0 - b2);
    float t0 = fminf(fdiv(tau, eps + b0), cap);
    float t1 = fminf(fdiv(tau, eps + b1), cap);
    float t2 = fminf(fdiv(tau, eps + b2), cap);
    float a0 = d0 * fmaf(t0, t0, 1.0f);
    float a1 = d1 * fmaf(t1, t1, 1.0f);
    float a2 = d2 * fmaf(t2, t2, 1.0f);
    float num = fmaf(a0, q0, fmaf(a1, q1, a2 * q2));
    return fdiv(num, a0 + a1 + a2);
}

// Left/right WENO5-Z at the interface between c2 and c3 (src/weno5.jl:25-61).
__device__ __forceinline__ void weno5_lr(float c0, float c1, float c2, float c3, float c4, float c5, float& L,
                                         float& R) {
    const float t13 = 1.0f / 3.0f, m76 = -7.0f / 6.0f, e116 = 11.0f / 6.0f, m16 = -1.0f / 6.0f, f56 = 5.0f / 6.0f;
    const float k1312 = 13.0f / 12.0f;
    // the same operations, multiply-adds and order as the two-lane weno5_lr2
    float qA = fmaf(e116, c2, fmaf(m76, c1, t13 * c0));
    float qB = fmaf(t13, c3, fmaf(f56, c2, m16 * c1));
    float qC = fmaf(m16, c4, fmaf(f56, c3, t13 * c2));
    float qD = fmaf(t13, c5, fmaf(m76, c4, e116 * c3));
    float s0 = fmaf(-2.0f, c1, c0) + c2, s1 = fmaf(-2.0f, c2, c1) + c3, s2 = fmaf(-2.0f, c3, c2) + c4,
          s3 = fmaf(-2.0f, c4, c3) + c5;
    float a = fmaf(3.0f, c2, fmaf(-4.0f, c1, c0));
    float b = c1 - c3;
    float c = fmaf(-4.0f, c3, 3.0f * c2) + c4;
    float d = fmaf(3.0f, c4, fmaf(-4.0f, c3, c2));
    float e = fmaf(-4.0f, c4, 3.0f * c3) + c5;
    float bA = fmaf(k1312 * s0, s0, 0.25f * a * a);
    float bB = fmaf(k1312 * s1, s1, 0.25f * b * b);
    float x2 = k1312 * s2 * s2;
    float bC = fmaf(0.25f * c, c, x2);
    float bD = fmaf(0.25f * d, d, x2);
    float bE = fmaf(k1312 * s3, s3, 0.25f * e * e);
    L = wz(bA, bB, bC, 0.1f, 0.6f, 0.3f, qA, qB, qC);
    R = wz(bB, bD, bE, 0.3f, 0.6f, 0.1f, qB, qC, qD);
}

// Two FP32 lanes in one 64-bit register pair.  sm_100's packed FP32
// instructions (add/sub/mul/fma .f32x2) issue once for both lanes, each lane
// rounding exactly as the scalar instruction would; the WENO5-Z arithmetic of
// two reconstructed fields runs this way (divisions, min and abs per lane).
struct f2 {
    unsigned long long v;
};
__device__ __forceinline__ f2 pk2(float a, float b) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void up2(f2 x, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x.v)); }
__device__ __forceinline__ f2 sp2(float a) { return pk2(a, a); }
__device__ __forceinline__ f2 operator+(f2 a, f2 b) {
    f2 d;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ f2 operator-(f2 a, f2 b) {
    f2 d;
    asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ f2 operator*(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return d;
}

// wz on two lanes: the same expressions as wz, lane by lane
__device__ __forceinline__ f2 wz2(f2 b0, f2 b1, f2 b2, float d0, float d1, float d2, f2 q0, f2 q1, f2 q2) {
    const float cap = 1e18f;
    const f2 eps = sp2(1e-36f), one = sp2(1.0f);
    f2 dt = b0 - b2;
    f2 e0 = eps + b0, e1 = eps + b1, e2 = eps + b2;
    float x, y, ex, ey;
    up2(dt, x, y);
    const float taux = fabsf(x), tauy = fabsf(y);
    up2(e0, ex, ey);
    f2 t0 = pk2(fminf(fdiv(taux, ex), cap), fminf(fdiv(tauy, ey), cap));
    up2(e1, ex, ey);
    f2 t1 = pk2(fminf(fdiv(taux, ex), cap), fminf(fdiv(tauy, ey), cap));
    up2(e2, ex, ey);
    f2 t2 = pk2(fminf(fdiv(taux, ex), cap), fminf(fdiv(tauy, ey), cap));
    f2 a0 = sp2(d0) * fma2(t0, t0, one);
    f2 a1 = sp2(d1) * fma2(t1, t1, one);
    f2 a2 = sp2(d2) * fma2(t2, t2, one);
    f2 num = fma2(a0, q0, fma2(a1, q1, a2 * q2));
    f2 den = a0 + a1 + a2;
    float nx, ny, dx, dy;
    up2(num, nx, ny);
    up2(den, dx, dy);
    return pk2(fdiv(nx, dx), fdiv(ny, dy));
}

// weno5_lr on two fields at once (lane 0 and lane 1 of every argument); the
// smoothness indicators bA..bE (left stencil: bA, bB, bC; right: bB, bD, bE)
// are returned for callers that test them
__device__ __forceinline__ void weno5_lr2(f2 c0, f2 c1, f2 c2, f2 c3, f2 c4, f2 c5, f2& L, f2& R, f2& bA, f2& bB,
                                          f2& bC, f2& bD, f2& bE) {
    const f2 t13 = sp2(1.0f / 3.0f), m76 = sp2(-7.0f / 6.0f), e116 = sp2(11.0f / 6.0f), m16 = sp2(-1.0f / 6.0f),
             f56 = sp2(5.0f / 6.0f), k1312 = sp2(13.0f / 12.0f), m2 = sp2(-2.0f), m4 = sp2(-4.0f), p3 = sp2(3.0f),
             q4 = sp2(0.25f);
    f2 qA = fma2(e116, c2, fma2(m76, c1, t13 * c0));
    f2 qB = fma2(t13, c3, fma2(f56, c2, m16 * c1));
    f2 qC = fma2(m16, c4, fma2(f56, c3, t13 * c2));
    f2 qD = fma2(t13, c5, fma2(m76, c4, e116 * c3));
    f2 s0 = fma2(m2, c1, c0) + c2, s1 = fma2(m2, c2, c1) + c3, s2 = fma2(m2, c3, c2) + c4,
       s3 = fma2(m2, c4, c3) + c5;
    f2 a = fma2(p3, c2, fma2(m4, c1, c0));
    f2 b = c1 - c3;
    f2 c = fma2(m4, c3, p3 * c2) + c4;
    f2 d = fma2(p3, c4, fma2(m4, c3, c2));
    f2 e = fma2(m4, c4, p3 * c3) + c5;
    bA = fma2(k1312 * s0, s0, q4 * a * a);
    bB = fma2(k1312 * s1, s1, q4 * b * b);
    f2 x2 = k1312 * s2 * s2;
    bC = fma2(q4 * c, c, x2);
    bD = fma2(q4 * d, d, x2);
    bE = fma2(k1312 * s3, s3, q4 * e * e);
    L = wz2(bA, bB, bC, 0.1f, 0.6f, 0.3f, qA, qB, qC);
    R = wz2(bB, bD, bE, 0.3f, 0.6f, 0.1f, qB, qC, qD);
}
__device__ __forceinline__ void weno5_lr2(f2 c0, f2 c1, f2 c2, f2 c3, f2 c4, f2 c5, f2& L, f2& R) {
    f2 bA, bB, bC, bD, bE;
    weno5_lr2(c0, c1, c2, c3, c4, c5, L, R, bA, bB, bC, bD, bE);
}

// f64::apply_floor with the FP64 pressure test skipped where an FP32
// estimate shows the cell far above both floors.  E - KE in FP32 is within
// ~1e-6 (|E| + KE) of its exact value, so a margin of 1e-5 (|E| + KE) above
// P_floor / (gamma - 1) means the FP64 test would change nothing; any cell
// below that margin, below the density floor or non-finite takes the FP64
// floor itself, so the result is apply_floor's in every case.
// true when the FP32 copy w of a cell (density v0 in FP64) shows it clear of
// both floors by that margin
__device__ __forceinline__ bool floor_clear(const float (&w)[5], double v0, double rho_floor, double Pfl_gm1) {
    if (!(v0 >= rho_floor)) return false;
    const float KE = fdiv(0.5f * fmaf(w[3], w[3], fmaf(w[2], w[2], w[1] * w[1])), w[0]);
    return w[4] - KE > fmaf(1e-5f, fabsf(w[4]) + KE, (float)Pfl_gm1);
}
__device__ __forceinline__ void floor_screened(double (&v)[5], double rho_floor, double P_floor, double Pfl_gm1,
                                               double gm1) {
    const float w[5] = {(float)v[0], (float)v[1], (float)v[2], (float)v[3], (float)v[4]};
    if (floor_clear(w, v[0], rho_floor, Pfl_gm1)) return;
    f64::apply_floor(v[0], v[1], v[2], v[3], v[4], rho_floor, P_floor, Pfl_gm1, gm1);
}
// A staged cell: the FP32 copy w of the floored state v (floors on active
// cells only), converting once where the cell is clear of the floors.
__device__ __forceinline__ void stage_floored(double (&v)[5], bool act, double rho_floor, double P_floor,
                                              double Pfl_gm1, double gm1, float (&w)[5]) {
#pragma unroll
    for (int q = 0; q < 5; ++q) w[q] = (float)v[q];
    if (!act || floor_clear(w, v[0], rho_floor, Pfl_gm1)) return;
    f64::apply_floor(v[0], v[1], v[2], v[3], v[4], rho_floor, P_floor, Pfl_gm1, gm1);
#pragma unroll
    for (int q = 0; q < 5; ++q) w[q] = (float)v[q];
}

__device__ __forceinline__ float cell_pressure(float r, float mx, float my, float mz, float E, float gm1) {
    r = fmaxf(r, 1e-30f);
    float KE = fdiv(0.5f * fmaf(mz, mz, fmaf(my, my, mx * mx)), r);
    return fmaxf(gm1 * (E - KE), 0.0f);
}

__device__ __forceinline__ float EL_from_P(float PL, float rL, float mx, float my, float mz, float inv_gm1) {
    float rp = fmaxf(rL, 1e-30f);
    float KE = fminf(fdiv(0.5f * fmaf(mz, mz, fmaf(my, my, mx * mx)), rp), 0.5f * rp * 1e4f);
    return fmaf(PL, inv_gm1, KE);
}

// HLLC (src/hllc.jl:17-165) in the rotated (normal, t1, t2) ordering.
__device__ __forceinline__ void hllc_normal(float rL, float mnL, float mt1L, float mt2L, float EL, float rR, float mnR,
                                            float mt1R, float mt2R, float ER, float g, float gm1, float gg,
                                            float F[5]) {
    if (rL <= 0.0f) { rL = 1e-30f; mnL = 0.0f; mt1L = 0.0f; mt2L = 0.0f; EL = 0.0f; }
    if (rR <= 0.0f) { rR = 1e-30f; mnR = 0.0f; mt1R = 0.0f; mt2R = 0.0f; ER = 0.0f; }
    rL = fmaxf(rL, 1e-30f);
    rR = fmaxf(rR, 1e-30f);
    float m2L = fmaf(mt2L, mt2L, fmaf(mt1L, mt1L, mnL * mnL));
    if (m2L > rL * rL * 1e4f) {
        float s = rL * 100.0f * rsqrtf(m2L);
        mnL *= s; mt1L *= s; mt2L *= s;
        m2L = fmaf(mt2L, mt2L, fmaf(mt1L, mt1L, mnL * mnL));
    }
    float m2R = fmaf(mt2R, mt2R, fmaf(mt1R, mt1R, mnR * mnR));
    if (m2R > rR * rR * 1e4f) {
        float s = rR * 100.0f * rsqrtf(m2R);
        mnR *= s; mt1R *= s; mt2R *= s;
        m2R = fmaf(mt2R, mt2R, fmaf(mt1R, mt1R, mnR * mnR));
    }
    float iL = fdiv(1.0f, rL), iR = fdiv(1.0f, rR);
    float KE_L = fminf(0.5f * m2L * iL, 0.5f * rL * 1e4f);
    float KE_R = fminf(0.5f * m2R * iR, 0.5f * rR * 1e4f);
    EL = fmaxf(EL, KE_L);
    ER = fmaxf(ER, KE_R);
    float vnL = mnL * iL, vt1L = mt1L * iL, vt2L = mt2L * iL;
    float vnR = mnR * iR, vt1R = mt1R * iR, vt2R = mt2R * iR;
    float pL = gm1 * (EL - KE_L), pR = gm1 * (ER - KE_R);
    float csL = sqrtf(g * pL * iL), csR = sqrtf(g * pR * iR);
    float SL, SR;
    if (pL > 0.0f && pR > 0.0f) {
        float r_avg = 0.5f * (rL + rR), cs_avg = 0.5f * (csL + csR);
        float p_star = fmaxf(0.0f, fmaf(-0.5f * (vnR - vnL) * r_avg, cs_avg, 0.5f * (pL + pR)));
        float qL = p_star > pL ? sqrtf(fmaf(gg, fdiv(p_star, pL) - 1.0f, 1.0f)) : 1.0f;
        float qR = p_star > pR ? sqrtf(fmaf(gg, fdiv(p_star, pR) - 1.0f, 1.0f)) : 1.0f;
        SL = fmaf(-csL, qL, vnL);
        SR = fmaf(csR, qR, vnR);
    } else {
        SL = fminf(vnL - csL, vnR - csR);
        SR = fmaxf(vnL + csL, vnR + csR);
    }
    float dL = rL * (SL - vnL), dR = rR * (SR - vnR);
    float denom = dL - dR;
    if (fabsf(denom) < 1e-36f) { F[0] = F[1] = F[2] = F[3] = F[4] = 0.0f; return; }
    float S_star = fdiv(fmaf(-mnR, SR - vnR, fmaf(mnL, SL - vnL, pR - pL)), denom);
    float FrL = mnL, FmnL = fmaf(mnL, vnL, pL), Fmt1L = mt1L * vnL, Fmt2L = mt2L * vnL, FEL = (EL + pL) * vnL;
    if (SL >= 0.0f) { F[0] = FrL; F[1] = FmnL; F[2] = Fmt1L; F[3] = Fmt2L; F[4] = FEL; return; }
    float FrR = mnR, FmnR = fmaf(mnR, vnR, pR), Fmt1R = mt1R * vnR, Fmt2R = mt2R * vnR, FER = (ER + pR) * vnR;
    if (SR <= 0.0f) { F[0] = FrR; F[1] = FmnR; F[2] = Fmt1R; F[3] = Fmt2R; F[4] = FER; return; }
    if (fmaxf(rL, rR) > 3.0f * fminf(rL, rR)) {
        float inv = fdiv(1.0f, SR - SL), SLSR = SL * SR;
        F[0] = fmaf(SLSR, rR - rL, fmaf(-SL, FrR, SR * FrL)) * inv;
        F[1] = fmaf(SLSR, mnR - mnL, fmaf(-SL, FmnR, SR * FmnL)) * inv;
        F[2] = fmaf(SLSR, mt1R - mt1L, fmaf(-SL, Fmt1R, SR * Fmt1L)) * inv;
        F[3] = fmaf(SLSR, mt2R - mt2L, fmaf(-SL, Fmt2R, SR * Fmt2L)) * inv;
        F[4] = fmaf(SLSR, ER - EL, fmaf(-SL, FER, SR * FEL)) * inv;
        return;
    }
    if (S_star >= 0.0f) {
        float chi = fdiv(dL, SL - S_star);
        float EsL = fabsf(dL) > 1e-36f ? chi * fmaf(S_star - vnL, S_star + fdiv(pL, dL), EL * iL) : 0.0f;
        F[0] = fmaf(SL, chi - rL, FrL);
        F[1] = fmaf(SL, fmaf(chi, S_star, -mnL), FmnL);
        F[2] = fmaf(SL, fmaf(chi, vt1L, -mt1L), Fmt1L);
        F[3] = fmaf(SL, fmaf(chi, vt2L, -mt2L), Fmt2L);
        F[4] = fmaf(SL, EsL - EL, FEL);
    } else {
        float chi = fdiv(dR, SR - S_star);
        float EsR = fabsf(dR) > 1e-36f ? chi * fmaf(S_star - vnR, S_star + fdiv(pR, dR), ER * iR) : 0.0f;
        F[0] = fmaf(SR, chi - rR, FrR);
        F[1] = fmaf(SR, fmaf(chi, S_star, -mnR), FmnR);
        F[2] = fmaf(SR, fmaf(chi, vt1R, -mt1R), Fmt1R);
        F[3] = fmaf(SR, fmaf(chi, vt2R, -mt2R), Fmt2R);
        F[4] = fmaf(SR, EsR - ER, FER);
    }
}

template <int D>
__device__ __forceinline__ void interface_flux(const float (&c)[6][6], float g, float gm1, float inv_gm1, float gg,
                                               float F[5]) {
    float L[5], R[5];
#pragma unroll
    for (int q = 0; q < 4; q += 2) {
        f2 L2, R2;
        weno5_lr2(pk2(c[0][q], c[0][q + 1]), pk2(c[1][q], c[1][q + 1]), pk2(c[2][q], c[2][q + 1]),
                  pk2(c[3][q], c[3][q + 1]), pk2(c[4][q], c[4][q + 1]), pk2(c[5][q], c[5][q + 1]), L2, R2);
        up2(L2, L[q], L[q + 1]);
        up2(R2, R[q], R[q + 1]);
    }
    float PL, PR;
    weno5_lr(c[0][5], c[1][5], c[2][5], c[3][5], c[4][5], c[5][5], PL, PR);
    float PmaxL = fmaxf(fmaxf(fmaxf(fmaxf(c[0][5], c[1][5]), c[2][5]), c[3][5]), c[4][5]);
    float PmaxR = fmaxf(fmaxf(fmaxf(fmaxf(c[1][5], c[2][5]), c[3][5]), c[4][5]), c[5][5]);
    PL = fminf(fmaxf(PL, 0.0f), PmaxL);
    PR = fminf(fmaxf(PR, 0.0f), PmaxR);
    float EL = EL_from_P(PL, L[0], L[1], L[2], L[3], inv_gm1);
    float ER = EL_from_P(PR, R[0], R[1], R[2], R[3], inv_gm1);
    float Fr[5];
    if (D == 0) {
        hllc_normal(L[0], L[1], L[2], L[3], EL, R[0], R[1], R[2], R[3], ER, g, gm1, gg, Fr);
        F[0] = Fr[0]; F[1] = Fr[1]; F[2] = Fr[2]; F[3] = Fr[3]; F[4] = Fr[4];
    } else if (D == 1) {
        hllc_normal(L[0], L[2], L[1], L[3], EL, R[0], R[2], R[1], R[3], ER, g, gm1, gg, Fr);
        F[0] = Fr[0]; F[1] = Fr[2]; F[2] = Fr[1]; F[3] = Fr[3]; F[4] = Fr[4];
    } else {
        hllc_normal(L[0], L[3], L[1], L[2], EL, R[0], R[3], R[1], R[2], ER, g, gm1, gg, Fr);
        F[0] = Fr[0]; F[1] = Fr[2]; F[2] = Fr[3]; F[3] = Fr[1]; F[4] = Fr[4];
    }
}

}  // namespace f32
}  // namespace bsn
