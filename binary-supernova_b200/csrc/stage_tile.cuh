// stage_tile.cuh -- the fused RK3-stage kernel as a template over the stencil
// physics (FP64 parity or FP32 fast) and the tile shape (chosen by the
// autotuner).  Included only by the translation units that instantiate it:
// hydro_f64.cu (FP64 physics, built with -fmad=false) and stage_fast.cu (FP32
// physics, built with FMA contraction and approximate division/sqrt).
//
// A CTA owns a TX x TY x TZ block of active cells.  For each sweep direction
// it stages the block plus a 3-cell halo along that direction in shared memory
// (SoA; floors applied in FP64 to active cells, ghost cells taken raw through
// the boundary map or from a ghost buffer, the cell pressure computed once per
// staged cell), computes every interface of the block once, and accumulates
// the flux divergence of its cells in FP64 registers.  The epilogue adds the
// source terms in the driver's order (BH gravity, self-gravity, sinks), the
// SSP-RK3 combine and the floors in FP64, stores the stage result and folds
// the next CFL speed into a device-wide max.
#pragma once

#include "stage_f64.cuh"
#include "tma.cuh"

namespace bsn {
namespace tile {

template <int TX, int TY, int TZ>
struct Shape {
    static constexpr int T[3] = {TX, TY, TZ};
    static constexpr int NCELL = TX * TY * TZ;
    static constexpr int EX0 = (TX + 6) * TY * TZ, EX1 = TX * (TY + 6) * TZ, EX2 = TX * TY * (TZ + 6);
    static constexpr int NEXT = EX0 > EX1 ? (EX0 > EX2 ? EX0 : EX2) : (EX1 > EX2 ? EX1 : EX2);
    static constexpr int FC0 = (TX + 1) * TY * TZ, FC1 = TX * (TY + 1) * TZ, FC2 = TX * TY * (TZ + 1);
    static constexpr int NFACE = FC0 > FC1 ? (FC0 > FC2 ? FC0 : FC2) : (FC1 > FC2 ? FC1 : FC2);
    // "cross" staging (all three sweeps from one staged region): the block,
    // then the 3-cell halos below/above it along x, y and z
    static constexpr int HX = 3 * TY * TZ, HY = 3 * TX * TZ, HZ = 3 * TX * TY;
    static constexpr int OXL = NCELL, OXH = OXL + HX, OYL = OXH + HX, OYH = OYL + HY, OZL = OYH + HY, OZH = OZL + HZ;
    static constexpr int NCROSS = OZH + HZ;
};

// Staged columns.  The stencils read rho, m_x, m_y, m_z and the cell pressure
// (c[s][0..3] and c[s][5]); E (c[s][4]) is staged only by policies whose
// epilogue reads the block's state back from shared memory (kCols = 6: E at
// column 4, P at 5).  With kCols = 5 the pressure sits in column 4.
template <int COLS>
__host__ __device__ constexpr int pcol() { return COLS - 1; }

// Physics policies --------------------------------------------------------
struct F64Physics {
    using real = double;
    static constexpr bool kStiffFallback = false;   // (already FP64)
    static constexpr bool kCross = true;             // stage the block and all halos once
    static constexpr bool kCenterFromSmem = true;   // smem holds the floored FP64 state
    static constexpr int kCols = 6;                 // staged columns: rho, m, E (read back by the epilogue), P
    static constexpr bool kWarpFaces = false;       // faces computed thread by thread
    static constexpr bool kQuiescentSkip = false;
    static constexpr bool kScreen = false;          // screening launch of a split stage
    __device__ static bool same(double, double) { return true; }
    static constexpr int kExtraSmem(int) { return 0; }
    __device__ static void prologue(unsigned char*, const f64::StageArgs&, int) {}
    struct Consts { double g, gm1; };
    __device__ static Consts consts(const f64::StageArgs& A) { return {A.g, A.gm1}; }
    // apply_floors (src/gpu_kernels.jl:26-46) on one cell, as the reference
    __device__ static void floor(double (&v)[5], const f64::StageArgs& A) {
        f64::apply_floor(v[0], v[1], v[2], v[3], v[4], A.rho_floor, A.P_floor, A.Pfl_gm1, A.gm1);
    }
    // a staged cell: floors on active cells, the staged copy
    __device__ static void stage(double (&v)[5], bool act, const f64::StageArgs& A, double (&w)[5]) {
        if (act) floor(v, A);
#pragma unroll
        for (int q = 0; q < 5; ++q) w[q] = v[q];
    }
    __device__ static double pressure(const double v[5], const Consts& k) {
        return f64::cell_pressure(v[0], v[1], v[2], v[3], v[4], k.gm1);
    }
    template <int D>
    __device__ static void flux(const double (&c)[6][6], const Consts& k, double F[5]) {
        f64::interface_flux<D>(c, k.g, k.gm1, F);
    }
};

// F32Physics (the fast path's policy) lives in stage_fast.cu.

__device__ __forceinline__ void load_cell(const f64::StageArgs& A, const Geom& G, int d, int a, int b, int c,
                                          double v[5], bool& active) {
    int n[3] = {G.nx, G.ny, G.nz};
    int p[3] = {a, b, c};
#pragma unroll
    for (int t = 0; t < 3; ++t)
        if (t != d) p[t] = p[t] < n[t] ? p[t] : n[t] - 1;   // partial tile: clamp (value unused)
    int pd = p[d];
    active = (pd >= 0 && pd < n[d]);
    const double* src = A.Uin;
    if (!active) {
        if (A.Gh) {
            pd = pd < -BSN_NG ? -BSN_NG : (pd > n[d] + BSN_NG - 1 ? n[d] + BSN_NG - 1 : pd);
            p[d] = pd;
            src = A.Gh;
        } else {
            p[d] = bc_map(pd, n[d], A.bc);
        }
    }
    long long off = G.act(p[0], p[1], p[2]);
#pragma unroll
    for (int q = 0; q < 5; ++q) v[q] = src[off + q];
}

// Staged values of the cross region (P::kCross) at entry e, from active
// coordinates (a, b, c) and the axis the cell may leave the grid along.
template <int TX, int TY, int TZ>
__device__ __forceinline__ void cross_cell(int e, int a0, int b0, int c0, const Geom& G, int& a, int& b, int& c,
                                           int& d) {
    using S = Shape<TX, TY, TZ>;
    if (e < S::OXL) {
        int i = e % TX, r = e / TX, j = r % TY, kk = r / TY;
        a = a0 + i; b = b0 + j; c = c0 + kk;
        d = a >= G.nx ? 0 : (b >= G.ny ? 1 : 2);   // partial block: the axis it leaves (used only along it)
    } else if (e < S::OYL) {
        int r = e - S::OXL;
        const bool hi = r >= S::HX;
        if (hi) r -= S::HX;
        int h = r % 3, rr = r / 3, j = rr % TY, kk = rr / TY;
        a = hi ? a0 + TX + h : a0 - 3 + h; b = b0 + j; c = c0 + kk; d = 0;
    } else if (e < S::OZL) {
        int r = e - S::OYL;
        const bool hi = r >= S::HY;
        if (hi) r -= S::HY;
        int i = r % TX, rr = r / TX, h = rr % 3, kk = rr / 3;
        a = a0 + i; b = hi ? b0 + TY + h : b0 - 3 + h; c = c0 + kk; d = 1;
    } else {
        int r = e - S::OZL;
        const bool hi = r >= S::HZ;
        if (hi) r -= S::HZ;
        int i = r % TX, rr = r / TX, j = rr % TY, h = rr / TY;
        a = a0 + i; b = b0 + j; c = hi ? c0 + TZ + h : c0 - 3 + h; d = 2;
    }
}

// Density contrast of a face's six-cell stencil above which a reduced-
// precision policy computes that face in FP64: where min rho < 1e-3 max rho
// the face states reconstructed on the thin side carry the rounding of the
// dense side's values (FP32: 1e-7 of them), i.e. relative errors of 1e-4 and
// more in the thin cell, whose velocity m / rho then runs away beside sinks.
constexpr float kStiffContrast = 1e-3f;

__device__ __forceinline__ bool stiff_stencil(const float (&c)[6][6]) {
    float lo = c[0][0], hi = c[0][0];
#pragma unroll
    for (int s = 1; s < 6; ++s) { lo = fminf(lo, c[s][0]); hi = fmaxf(hi, c[s][0]); }
    return lo < kStiffContrast * hi;
}

// The FP64 flux of the face between active cells p_D - 1 and p_D along D
// (p: the face's cell on the high side), from the FP64 state as the FP64
// path stages it (boundary map, floors on active cells, pressure once):
// the same operations, so the same bits as the FP64 path's flux there.
template <int D>
__device__ __noinline__ void face_flux_f64(const f64::StageArgs& A, int a, int b, int c, double F[5]) {
    Geom G(A.nx, A.ny, A.nz);
    double cs[6][6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        int p[3] = {a, b, c};
        p[D] += s - 3;
        double v[5];
        bool act;
        load_cell(A, G, D, p[0], p[1], p[2], v, act);
        if (act) f64::apply_floor(v[0], v[1], v[2], v[3], v[4], A.rho_floor, A.P_floor, A.Pfl_gm1, A.gm1);
#pragma unroll
        for (int q = 0; q < 5; ++q) cs[s][q] = v[q];
        cs[s][5] = f64::cell_pressure(v[0], v[1], v[2], v[3], v[4], A.gm1);
    }
    f64::interface_flux<D>(cs, A.g, A.gm1, F);
}

template <class P, int TX, int TY, int TZ, int NT, int D, bool LED>
__device__ void sweep(const f64::StageArgs& A, const Geom& G, const typename P::Consts& k, int a0, int b0, int c0,
                      typename P::real* sC, typename P::real* sF, unsigned char* psm,
                      double (&acc)[Shape<TX, TY, TZ>::NCELL / NT][5], bool quiet_cross, double* sled) {
    constexpr bool CROSS = P::kCross;
    using S = Shape<TX, TY, TZ>;
    using real = typename P::real;
    constexpr int CPT = S::NCELL / NT;
    constexpr int LX = TX + (D == 0 ? 6 : 0), LY = TY + (D == 1 ? 6 : 0), LZ = TZ + (D == 2 ? 6 : 0);
    constexpr int FX = TX + (D == 0), FY = TY + (D == 1), FZ = TZ + (D == 2);
    constexpr int NE = LX * LY * LZ, NF = FX * FY * FZ;
    constexpr int TD = D == 0 ? TX : (D == 1 ? TY : TZ);
    const int tid = threadIdx.x;
    const int n[3] = {G.nx, G.ny, G.nz};
    const int o[3] = {a0, b0, c0};

    bool quiet = false;
    if constexpr (CROSS) {
        __syncthreads();   // staged once by stage_block; sF free after the previous sweep's divergence
    } else {
        __syncthreads();
        for (int e = tid; e < NE; e += NT) {
            int ex = e % LX, r = e / LX, ey = r % LY, ez = r / LY;
            int a = a0 + ex - (D == 0 ? 3 : 0);
            int b = b0 + ey - (D == 1 ? 3 : 0);
            int c = c0 + ez - (D == 2 ? 3 : 0);
            double v[5];
            bool act;
            load_cell(A, G, D, a, b, c, v, act);
            real w[5];
            P::stage(v, act, A, w);
#pragma unroll
            for (int q = 0; q < 5; ++q)
                if (q < 4 || P::kCols == 6) sC[q * S::NEXT + e] = w[q];
            sC[pcol<P::kCols>() * S::NEXT + e] = P::pressure(w, k);
        }
        // policies with per-stencil work that only non-uniform data can need
        // (the learned weights' fallback test) learn here whether every staged
        // value of the sweep equals the first one within the policy's margin
        if constexpr (P::kQuiescentSkip) {
            __syncthreads();
            bool varied = false;
            for (int e = tid; e < NE; e += NT) {
#pragma unroll
                for (int q = 0; q < 5; ++q) {   // rho, m, P (E is not reconstructed)
                    const int col = q < 4 ? q : pcol<P::kCols>();
                    varied |= !P::same(sC[col * S::NEXT + e], sC[col * S::NEXT]);
                }
            }
            quiet = !__syncthreads_or(varied);
        } else {
            __syncthreads();
        }
    }
    if constexpr (CROSS) quiet = quiet_cross;
    constexpr int SD = (D == 0) ? 1 : (D == 1 ? LX : LX * LY);
    constexpr int FSTR = CROSS ? S::NCROSS : S::NEXT;   // field stride of the staged values
    // staged index of stencil cell s (0..5, cells fd-3 .. fd+2 along D) of face (fx, fy, fz)
    auto sidx = [&](int fx, int fy, int fz, int s) -> int {
        if constexpr (!CROSS) {
            return fx + LX * (fy + LY * fz) + s * SD;
        } else {
            const int fd = D == 0 ? fx : (D == 1 ? fy : fz);
            const int p = fd - 3 + s;
            int cb, cs, lo, hs;
            if (D == 0) { cb = TX * (fy + TY * fz); cs = 1; lo = S::OXL + 3 * (fy + TY * fz); hs = 1; }
            else if (D == 1) { cb = fx + TX * TY * fz; cs = TX; lo = S::OYL + fx + 3 * TX * fz; hs = TX; }
            else { cb = fx + TX * fy; cs = TX * TY; lo = S::OZL + fx + TX * fy; hs = TX * TY; }
            constexpr int H = D == 0 ? S::HX : (D == 1 ? S::HY : S::HZ);
            return p < 0 ? lo + (p + 3) * hs : (p < TD ? cb + p * cs : lo + H + (p - TD) * hs);
        }
    };
    // one face: write it to smem and, if this tile owns it, to the optional
    // flux arrays, coarse flux registers and fine boundary-face buffers
    auto emit = [&](int f, int fx, int fy, int fz, const real (&F)[5]) {
#pragma unroll
        for (int q = 0; q < 5; ++q) sF[q * S::NFACE + f] = F[q];
        int fpos[3] = {fx, fy, fz};
        int gd = o[D] + fpos[D];
        bool owner = (fpos[D] < TD) || (gd == n[D]);
        if (!owner) return;
        int ga = o[0] + fx, gb = o[1] + fy, gc = o[2] + fz;
        if (A.F[D]) {
            long long ex_ = (G.nx + 2 * BSN_NG) + (D == 0), ey_ = (G.ny + 2 * BSN_NG) + (D == 1);
            long long ii = ga + BSN_NG - (D == 0), jj = gb + BSN_NG - (D == 1), kk = gc + BSN_NG - (D == 2);
            long long off = 5LL * (ii + ex_ * (jj + ey_ * kk));
#pragma unroll
            for (int q = 0; q < 5; ++q) A.F[D][off + q] = (double)F[q];
        }
        if (A.use_reg) {
            const f64::RegFaces& R = A.reg;
            int ta = (D == 0) ? gb : ga, tb = (D == 2) ? gb : gc;
            int ax1 = (D == 0) ? 1 : 0, ax2 = (D == 2) ? 1 : 2;
            if (ta >= R.t0[ax1] && ta <= R.t1[ax1] && tb >= R.t0[ax2] && tb <= R.t1[ax2]) {
                int n1 = R.t1[ax1] - R.t0[ax1] + 1;
                long long roff = 5LL * ((ta - R.t0[ax1]) + (long long)n1 * (tb - R.t0[ax2]));
                double* dst = nullptr;
                if (gd == R.lo[D]) dst = R.reg[2 * D];
                else if (gd == R.hi[D]) dst = R.reg[2 * D + 1];
                if (dst) {
                    double fac = A.dt_dev ? A.reg.wt * *A.dt_dev : R.fac;
#pragma unroll
                    for (int q = 0; q < 5; ++q) dst[roff + q] += fac * (double)F[q];
                }
            }
        }
        if (LED && A.ledger && A.led_bnd && (gd == 0 || gd == n[D])) {   // mass through the grid's boundary
            // per unit volume, as the divergence sees it (the flush multiplies by dV)
            const double inv = (D == 0) ? A.idx : (D == 1 ? A.idy : A.idz);
            atomicAdd(&sled[f64::LED_BND], (gd == 0 ? (double)F[0] : -(double)F[0]) * inv);
        }
        if (A.use_bnd && (gd == 0 || gd == n[D])) {
            int ta = (D == 0) ? gb : ga, tb = (D == 2) ? gb : gc;
            int n1 = (D == 0) ? G.ny : G.nx;
            long long roff = 5LL * (ta + (long long)n1 * tb);
            double* dst = A.bnd.f[2 * D + (gd == 0 ? 0 : 1)];
#pragma unroll
            for (int q = 0; q < 5; ++q) dst[roff + q] = (double)F[q];
        }
    };
    auto face_valid = [&](int fx, int fy, int fz) {
        int fpos[3] = {fx, fy, fz};
        bool valid = true;
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            int gpos = o[t] + fpos[t];
            valid = valid && (t == D ? gpos <= n[t] : gpos < n[t]);
        }
        return valid;
    };
    // thread-per-face loop (the plain stencil physics); faces whose density
    // stencil is stiff (kStiffFallback policies) are listed for a second pass
    // that computes them in FP64, so the main loop keeps its registers, and
    // the listed faces are spread over all threads of the block (they
    // cluster: a star's surface, a sink's surroundings)
    __shared__ int s_nstiff;
    __shared__ int s_stiff[P::kStiffFallback ? NF : 1];
    auto plain_faces = [&]() {
        if constexpr (P::kStiffFallback) {
            if (tid == 0) s_nstiff = 0;
            __syncthreads();
        }
        for (int f = tid; f < NF; f += NT) {
            int fx = f % FX, r = f / FX, fy = r % FY, fz = r / FY;
            if (!face_valid(fx, fy, fz)) continue;
            real c[6][6];
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                const int e = sidx(fx, fy, fz, s);
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    const int col = q < 4 ? q : (q == 5 ? pcol<P::kCols>() : 4);
                    c[s][q] = (q == 4 && P::kCols == 5) ? (real)0 : sC[col * FSTR + e];
                }
            }
            if constexpr (P::kStiffFallback) {
                if (stiff_stencil(c)) { s_stiff[atomicAdd(&s_nstiff, 1)] = f; continue; }
            }
            real F[5];
            P::template flux<D>(c, k, F);
            emit(f, fx, fy, fz, F);
        }
        if constexpr (P::kStiffFallback) {
            __syncthreads();
            const int nst = s_nstiff;   // read by every thread before the next sweep resets it
            for (int i = tid; i < nst; i += NT) {
                const int f = s_stiff[i];
                const int fx = f % FX, r = f / FX, fy = r % FY, fz = r / FY;
                double F64[5];
                face_flux_f64<D>(A, o[0] + fx, o[1] + fy, o[2] + fz, F64);
                real F[5];
#pragma unroll
                for (int q = 0; q < 5; ++q) F[q] = (real)F64[q];
                emit(f, fx, fy, fz, F);
            }
        }
    };
    if constexpr (P::kWarpFaces) {
        if (P::kQuiescentSkip && quiet) {
            plain_faces();   // uniform sweep: no per-stencil work can apply, the policy's plain flux
        } else {
            // warp-collective faces (tensor-core work inside the flux): every
            // lane of a warp takes part in every iteration, valid face or not
            const int warp = tid >> 5, lane = tid & 31;
            for (int fb = warp * 32; fb < NF; fb += NT) {
                int f = fb + lane;
                int fx = f % FX, r = f / FX, fy = r % FY, fz = r / FY;
                bool valid = f < NF && face_valid(fx, fy, fz);
                real c[6][6];
#pragma unroll
                for (int s = 0; s < 6; ++s) {
                    const int e = valid ? sidx(fx, fy, fz, s) : 0;
#pragma unroll
                    for (int q = 0; q < 6; ++q) {
                        const int col = q < 4 ? q : (q == 5 ? pcol<P::kCols>() : 4);
                        c[s][q] = (valid && (q != 4 || P::kCols == 6)) ? sC[col * FSTR + e] : (real)0;
                    }
                }
                real F[5];
                P::template warp_flux<D>(c, valid, k, F, psm, warp, quiet);
                if (valid) emit(f, fx, fy, fz, F);
            }
        }
    } else {
        plain_faces();
    }
    __syncthreads();

    const double inv = (D == 0) ? A.idx : (D == 1 ? A.idy : A.idz);
    constexpr int FS = (D == 0) ? 1 : (D == 1 ? FX : FX * FY);
#pragma unroll
    for (int m = 0; m < CPT; ++m) {
        int cell = tid + m * NT;
        int i = cell % TX, j = (cell / TX) % TY, kk = cell / (TX * TY);
        int fl = i + FX * (j + FY * kk);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            double dF = (double)sF[q * S::NFACE + fl + FS] - (double)sF[q * S::NFACE + fl];
            if (D == 0) acc[m][q] = -dF * inv;
            else acc[m][q] = acc[m][q] - dF * inv;
        }
    }
}

// Policy-specific shared memory (learned parameters, row buffers) after the
// staged cells and faces.
template <class P, int TX, int TY, int TZ>
__device__ __forceinline__ unsigned char* policy_smem(unsigned char* smem_raw) {
    using S = Shape<TX, TY, TZ>;
    constexpr int NST = P::kCross ? S::NCROSS : S::NEXT;
    return smem_raw + ((sizeof(typename P::real) * (P::kCols * NST + 5 * S::NFACE) + 15) / 16) * 16;
}

// Whether active cell (a, b, c) counts in the mass ledger: outside the
// region a finer level covers (half-open [led_skip_lo, led_skip_hi)).
__device__ __forceinline__ bool led_counted(const f64::StageArgs& A, int a, int b, int c) {
    return !(a >= A.led_skip_lo[0] && a < A.led_skip_hi[0] && b >= A.led_skip_lo[1] && b < A.led_skip_hi[1] &&
             c >= A.led_skip_lo[2] && c < A.led_skip_hi[2]);
}

// TMA staging state of a CTA (stage_kernel_tma): the tensor maps, the two
// raw buffers, their mbarriers and the parity each barrier completes next.
struct TmaCtx {
    const tma::Maps* M;
    double* raw[2];
    uint64_t* bar;
    uint32_t ph[2];
};

// Raw-buffer placement of a tile: inside the face buffer when it is free
// (it is during staging) and large enough, else after the policy's smem.
// Copies of kChunkCap bytes where the dynamic smem still fits MINB CTAs per
// SM, else copies small enough for both buffers to sit in the face buffer.
template <class P, int TX, int TY, int TZ, int NT, int MINB>
struct TmaSmem {
    using S = Shape<TX, TY, TZ>;
    static constexpr int FACE_OFF = (int)sizeof(typename P::real) * P::kCols * S::NCROSS;
    static constexpr int FACE_BYTES = (int)sizeof(typename P::real) * 5 * S::NFACE;
    static constexpr int APPEND_OFF = (int)(((sizeof(typename P::real) * (P::kCols * S::NCROSS + 5 * S::NFACE) + 16) +
                                             127) / 128 * 128);
    static constexpr int in_faces(int rawb) { return FACE_BYTES >= 2 * rawb ? 2 : (FACE_BYTES >= rawb ? 1 : 0); }
    static constexpr int bytes_for(int rawb) { return APPEND_OFF + (2 - in_faces(rawb)) * rawb; }
    static constexpr int BUDGET = 233472 / MINB - 2048;   // per-CTA smem that keeps MINB CTAs on an SM
    static constexpr int CAP = bytes_for(tma::Chunks<TX, TY, TZ, tma::kChunkCap>::RAWB) <= BUDGET
                                   ? tma::kChunkCap
                                   : FACE_BYTES / 2 / 128 * 128;
    using C = tma::Chunks<TX, TY, TZ, CAP>;
    static constexpr int IN_FACES = in_faces(C::RAWB);
    static constexpr int BYTES = bytes_for(C::RAWB);   // dynamic smem of the TMA kernel
    static_assert(FACE_OFF % 128 == 0, "face buffer must start on a 128-byte boundary for TMA copies");
    // raw buffer 0 always lies in the face buffer (the layouts this path is
    // verified with); a tile whose copies fit only after the face buffer
    // keeps the plain loader
    static constexpr bool OK = IN_FACES >= 1;
};

// The cross region of block (a0, b0, c0) staged by TMA copies: each copy's
// cells converted as the plain loader converts them (P::stage, pressure),
// cells outside the active domain through the boundary map instead.  Returns
// false on every thread when a copy did not arrive within the wait bound
// (the error word is set and the copies in flight are waited for, bounded).
template <class P, int TX, int TY, int TZ, int NT, int MINB>
__device__ bool stage_cross_tma(const f64::StageArgs& A, TmaCtx& T, const Geom& G, const typename P::Consts& k,
                                int a0, int b0, int c0, typename P::real* sC) {
    using S = Shape<TX, TY, TZ>;
    using C = typename TmaSmem<P, TX, TY, TZ, NT, MINB>::C;
    using real = typename P::real;
    const int tid = threadIdx.x;
    const tma::Maps& M = *T.M;
    const int n[3] = {G.nx, G.ny, G.nz};
    auto issue = [&](int c, int b) {   // thread 0: copy c into buffer b
        uint32_t bytes;
        const CUtensorMap* map;
        int x, y, z;
        if (c < C::NA) {
            map = &M.a; bytes = C::BA; x = 5 * a0;
            y = b0 + 3 + (c % C::NAY) * C::AY; z = c0 + 3 + (c / C::NAY) * C::AZ;
        } else if (c < C::NA + C::NY) {
            const int r = c - C::NA, hi = r >= C::NY / 2, p = hi ? r - C::NY / 2 : r;
            map = &M.y; bytes = C::BY; x = 5 * (a0 + 2); y = hi ? b0 + TY + 3 : b0; z = c0 + 3 + p * C::YZ;
        } else {
            const int r = c - C::NA - C::NY, hi = r >= C::NZ / 2, p = hi ? r - C::NZ / 2 : r;
            map = &M.z; bytes = C::BZ; x = 5 * (a0 + 2); y = b0 + 3 + p * C::ZY; z = hi ? c0 + TZ + 3 : c0;
        }
        tma::fence_proxy_async();   // earlier generic accesses of the buffer before the copy's writes
        tma::mbar_expect_tx(&T.bar[b], bytes);
        tma::load_3d(T.raw[b], map, &T.bar[b], x, y, z);
    };
    // one staged cell: from the copy (src, 5 doubles) when it lies in the
    // active domain along axis d, else through the boundary map
    auto put = [&](int e, int a, int b, int c, int d, const double* src) {
        const int p = d == 0 ? a : (d == 1 ? b : c);
        double v[5];
        bool act = true;
        if (p >= 0 && p < n[d]) {
#pragma unroll
            for (int q = 0; q < 5; ++q) v[q] = src[q];
        } else {
            load_cell(A, G, d, a, b, c, v, act);
        }
        real w[5];
        P::stage(v, act, A, w);
#pragma unroll
        for (int q = 0; q < 5; ++q)
            if (q < 4 || P::kCols == 6) sC[q * S::NCROSS + e] = w[q];
        sC[pcol<P::kCols>() * S::NCROSS + e] = P::pressure(w, k);
    };
    if (tid == 0) {
        issue(0, 0);
        if (C::N > 1) issue(1, 1);
    }
    for (int c = 0; c < C::N; ++c) {
        const int b = c & 1;
        const bool got = tma::mbar_wait_bounded(&T.bar[b], T.ph[b]);
        const double* raw = T.raw[b];
        if (got) {
            if (c < C::NA) {   // block rows with their x halos: AY rows x AZ planes
                const int j0 = (c % C::NAY) * C::AY, k0 = (c / C::NAY) * C::AZ;
                for (int t = tid; t < (TX + 6) * C::AY * C::AZ; t += NT) {
                    const int ib = t % (TX + 6), r = t / (TX + 6), jb = r % C::AY, kb = r / C::AY;
                    const int j = j0 + jb, kk = k0 + kb;
                    const int e = ib < 3 ? S::OXL + ib + 3 * (j + TY * kk)
                                         : (ib >= TX + 3 ? S::OXH + (ib - TX - 3) + 3 * (j + TY * kk)
                                                         : (ib - 3) + TX * (j + TY * kk));
                    put(e, a0 - 3 + ib, b0 + j, c0 + kk, 0, raw + 5 * ib + C::RA * (jb + C::AY * kb));
                }
            } else if (c < C::NA + C::NY) {   // y halo rows
                const int r = c - C::NA, hi = r >= C::NY / 2, p = hi ? r - C::NY / 2 : r;
                for (int t = tid; t < TX * 3 * C::YZ; t += NT) {
                    const int i = t % TX, r2 = t / TX, h = r2 % 3, kb = r2 / 3, kk = p * C::YZ + kb;
                    const int e = (hi ? S::OYH : S::OYL) + i + TX * (h + 3 * kk);
                    put(e, a0 + i, hi ? b0 + TY + h : b0 - 3 + h, c0 + kk, 1, raw + 5 * (i + 1) + C::RH * (h + 3 * kb));
                }
            } else {   // z halo planes
                const int r = c - C::NA - C::NY, hi = r >= C::NZ / 2, p = hi ? r - C::NZ / 2 : r;
                for (int t = tid; t < TX * C::ZY * 3; t += NT) {
                    const int i = t % TX, r2 = t / TX, jb = r2 % C::ZY, h = r2 / C::ZY, j = p * C::ZY + jb;
                    const int e = (hi ? S::OZH : S::OZL) + i + TX * (j + TY * h);
                    put(e, a0 + i, b0 + j, hi ? c0 + TZ + h : c0 - 3 + h, 2,
                        raw + 5 * (i + 1) + C::RH * (jb + C::ZY * h));
                }
            }
        }
        // every thread is done with buffer b; one decision for the whole CTA
        const bool ok = __syncthreads_and(got);
        if (!ok) {
            if (tid == 0) {
                if (M.err) atomicOr(M.err, 1u);
                // the copies still in flight: this one and the other buffer's
                tma::mbar_wait_bounded(&T.bar[b], T.ph[b]);
                if (c + 1 < C::N) tma::mbar_wait_bounded(&T.bar[b ^ 1], T.ph[b ^ 1]);
            }
            __syncthreads();
            return false;
        }
        T.ph[b] ^= 1u;
        if (tid == 0 && c + 2 < C::N) issue(c + 2, b);
    }
    return true;
}

// One RK3 stage (or euler3d_rhs!) of the TX x TY x TZ block at active
// origin (a0, b0, c0): three sweeps, sources, combine, floors, CFL fold.
// Starts with a barrier (the first sweep's), so a CTA may call it for one
// block after another.
template <class P, int TX, int TY, int TZ, int NT, int MINB = 1, bool LED = false>
__device__ __forceinline__ bool stage_block(const f64::StageArgs& A, int a0, int b0, int c0,
                                            unsigned char* smem_raw, double* red, unsigned int& nanflag,
                                            TmaCtx* T = nullptr) {
    using S = Shape<TX, TY, TZ>;
    using real = typename P::real;
    static_assert(S::NCELL % NT == 0, "cells must divide evenly among threads");
    constexpr int CPT = S::NCELL / NT;
    real* sC = reinterpret_cast<real*>(smem_raw);
    real* sF = sC + P::kCols * (P::kCross ? S::NCROSS : S::NEXT);

    Geom G(A.nx, A.ny, A.nz);
    const int tid = threadIdx.x;
    if (tid == 0) nanflag = 0;
    const typename P::Consts k = P::consts(A);
    unsigned char* psm = policy_smem<P, TX, TY, TZ>(smem_raw);
    double acc[CPT][5];
    // this block's mass-ledger sums (LED kernels with A.ledger set; the other
    // kernels carry no ledger code at all)
    __shared__ double sled[LED ? f64::LED_TERMS : 1];
    if (LED && A.ledger && tid < f64::LED_TERMS) sled[tid] = 0.0;   // ordered before use by the staging barriers
    if constexpr (P::kCross) {
        // the block and the halos of all three sweeps, staged once (floors in
        // FP64 on active cells, ghosts raw, pressure once per cell)
        __syncthreads();   // the previous block of a persistent CTA is done with smem
        if (T) {
            if (!stage_cross_tma<P, TX, TY, TZ, NT, MINB>(A, *T, G, k, a0, b0, c0, sC)) return false;
        } else {
            for (int e = tid; e < S::NCROSS; e += NT) {
                int a, b, c, d;
                cross_cell<TX, TY, TZ>(e, a0, b0, c0, G, a, b, c, d);
                double v[5];
                bool act;
                load_cell(A, G, d, a, b, c, v, act);
                real w[5];
                P::stage(v, act, A, w);
#pragma unroll
                for (int q = 0; q < 5; ++q)
                    if (q < 4 || P::kCols == 6) sC[q * S::NCROSS + e] = w[q];
                sC[pcol<P::kCols>() * S::NCROSS + e] = P::pressure(w, k);
            }
        }
    }
    // policies with per-stencil work that only non-uniform data can need (the
    // learned weights' fallback test) learn here, per sweep, whether every
    // value the sweep's stencils read (the block and that sweep's halos)
    // equals the block's first cell within the policy's margin
    bool quiet[3] = {false, false, false};
    if constexpr (P::kCross && P::kQuiescentSkip) {
        __syncthreads();
        unsigned varied = 0u;   // bit 0: block, bits 1-3: x, y, z halos
        for (int e = tid; e < S::NCROSS; e += NT) {
            bool v = false;
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const int col = q < 4 ? q : pcol<P::kCols>();
                v |= !P::same(sC[col * S::NCROSS + e], sC[col * S::NCROSS]);
            }
            if (v) varied |= e < S::OXL ? 1u : (e < S::OYL ? 2u : (e < S::OZL ? 4u : 8u));
        }
        const bool vb = __syncthreads_or(varied & 1u), vx = __syncthreads_or(varied & 2u),
                   vy = __syncthreads_or(varied & 4u), vz = __syncthreads_or(varied & 8u);
        quiet[0] = !(vb || vx);
        quiet[1] = !(vb || vy);
        quiet[2] = !(vb || vz);
        if constexpr (P::kScreen) {
            // a block with a non-uniform sweep is left to the split stage's
            // other launch: listed, nothing written here (the test is uniform
            // over the CTA, so every thread returns)
            if (!(quiet[0] && quiet[1] && quiet[2])) {
                if (tid == 0) {
                    const int gx = (A.nx + TX - 1) / TX, gy = (A.ny + TY - 1) / TY;
                    A.split_list[atomicAdd(A.split_count, 1u)] = a0 / TX + gx * (b0 / TY + gy * (c0 / TZ));
                }
                return true;
            }
        }
    }
    sweep<P, TX, TY, TZ, NT, 0, LED>(A, G, k, a0, b0, c0, sC, sF, psm, acc, quiet[0], sled);
    sweep<P, TX, TY, TZ, NT, 1, LED>(A, G, k, a0, b0, c0, sC, sF, psm, acc, quiet[1], sled);
    sweep<P, TX, TY, TZ, NT, 2, LED>(A, G, k, a0, b0, c0, sC, sF, psm, acc, quiet[2], sled);

    const double dt = A.dt_dev ? *A.dt_dev : A.dt;
    const f64::BHSrc& BH = A.bh_dev ? *A.bh_dev : A.bh;     // kernel parameters are __grid_constant__
    const f64::SinkSrc& SK = A.sk_dev ? *A.sk_dev : A.sk;
    const double cdt = A.stage == 2 ? 0.25 * dt : (A.stage == 3 ? (2.0 / 3.0) * dt : dt);
    double smax = 0.0;
#pragma unroll
    for (int m = 0; m < CPT; ++m) {
        int cell = tid + m * NT;
        int i = cell % TX, j = (cell / TX) % TY, kk = cell / (TX * TY);
        int a = a0 + i, b = b0 + j, c = c0 + kk;
        if (a >= A.nx || b >= A.ny || c >= A.nz) continue;
        long long off = G.act(a, b, c);
        double u0, u1, u2, u3, u4;
        if (P::kCenterFromSmem) {
            // the block's cells: the cross region's first part, or the z-extended block of the last sweep
            constexpr int FS = P::kCross ? S::NCROSS : S::NEXT;
            int e = P::kCross ? i + TX * (j + TY * kk) : i + TX * (j + TY * (kk + 3));
            u0 = (double)sC[0 * FS + e]; u1 = (double)sC[1 * FS + e]; u2 = (double)sC[2 * FS + e];
            u3 = (double)sC[3 * FS + e]; u4 = (double)sC[4 * FS + e];
        } else {
            double v[5] = {A.Uin[off], A.Uin[off + 1], A.Uin[off + 2], A.Uin[off + 3], A.Uin[off + 4]};
            P::floor(v, A);
            u0 = v[0]; u1 = v[1]; u2 = v[2]; u3 = v[3]; u4 = v[4];
        }
        double* d = acc[m];
        double xc = A.x0 + ((double)(a + 1) - 0.5) * A.dx;
        double yc = A.y0 + ((double)(b + 1) - 0.5) * A.dy;
        double zc = A.z0 + ((double)(c + 1 + A.k0) - 0.5) * A.dz;
        if (A.use_bh) {   // src/gpu_kernels.jl:199-230
            double vx = u1 / u0, vy = u2 / u0, vz = u3 / u0;
            double ax = 0.0, ay = 0.0, az = 0.0;
            for (int nb = 0; nb < BH.n; ++nb) {
                double ddx = xc - BH.px[nb], ddy = yc - BH.py[nb], ddz = zc - BH.pz[nb];
                double r2 = sq(ddx) + sq(ddy) + sq(ddz) + sq(BH.eps[nb]);
                double r3 = r2 * sqrt(r2);
                double fac = -BH.mass[nb] / r3;
                ax += fac * ddx; ay += fac * ddy; az += fac * ddz;
            }
            d[1] += u0 * ax; d[2] += u0 * ay; d[3] += u0 * az;
            d[4] += u0 * (vx * ax + vy * ay + vz * az);
        }
        if (A.use_sg) {   // src/gpu_kernels.jl:291-319
            int nx = A.nx, ny = A.ny, nz = A.nz;
            int ip = min(a + 1, nx - 1), im = max(a - 1, 0);
            int jp = min(b + 1, ny - 1), jm = max(b - 1, 0);
            int kp = min(c + 1, nz - 1), km = max(c - 1, 0);
            double fx = ip > im ? A.inv2dx : 2.0 * A.inv2dx;
            double fy = jp > jm ? A.inv2dy : 2.0 * A.inv2dy;
            double fz = kp > km ? A.inv2dz : 2.0 * A.inv2dz;
            const double* Pp = A.phi;
            long long sy = nx, sz = (long long)nx * ny;
            double gx = (Pp[ip + sy * b + sz * c] - Pp[im + sy * b + sz * c]) * fx;
            double gy = (Pp[a + sy * jp + sz * c] - Pp[a + sy * jm + sz * c]) * fy;
            double pzp = Pp[a + sy * b + sz * kp], pzm = Pp[a + sy * b + sz * km];
            if (A.phi_lo || A.phi_hi) {   // a slab's edge planes: the larger grid's central difference
                fz = A.inv2dz;
                if (c == nz - 1 && A.phi_hi) pzp = A.phi_hi[a + sy * b];
                if (c == 0 && A.phi_lo) pzm = A.phi_lo[a + sy * b];
            }
            double gz = (pzp - pzm) * fz;
            double vdotg = (u1 * gx + u2 * gy + u3 * gz) / u0;
            d[1] -= u0 * gx; d[2] -= u0 * gy; d[3] -= u0 * gz; d[4] -= u0 * vdotg;
        }
        if (A.use_sink && u0 > SK.rho_min) {   // src/gpu_kernels.jl:238-284
            for (int nb = 0; nb < SK.n; ++nb) {
                double ddx = xc - SK.px[nb], ddy = yc - SK.py[nb], ddz = zc - SK.pz[nb];
                double rr = sqrt(sq(ddx) + sq(ddy) + sq(ddz));
                if (rr < SK.rs[nb]) {
                    double ts = SK.ts[nb];
                    d[0] -= u0 / ts;
                    if (LED && A.ledger && led_counted(A, a, b, c)) atomicAdd(&sled[f64::LED_DRAIN], u0 / ts);
                    if (SK.torque_free) {
                        double rx = ddx / rr, ry = ddy / rr, rz = ddz / rr;
                        double vx = u1 / u0, vy = u2 / u0, vz = u3 / u0;
                        double vrx = vx - SK.vx[nb], vry = vy - SK.vy[nb], vrz = vz - SK.vz[nb];
                        double v_r = vrx * rx + vry * ry + vrz * rz;
                        double e_int = u4 / u0 - 0.5 * (sq(vx) + sq(vy) + sq(vz));
                        d[1] -= u0 * v_r * rx / ts;
                        d[2] -= u0 * v_r * ry / ts;
                        d[3] -= u0 * v_r * rz / ts;
                        d[4] -= (0.5 * u0 * sq(v_r) + u0 * e_int) / ts;
                    } else {
                        d[1] -= u1 / ts; d[2] -= u2 / ts; d[3] -= u3 / ts; d[4] -= u4 / ts;
                    }
                }
            }
        }
        if (A.use_rot) f64::rot_frame_src(d, u0, u1, u2, xc, yc, A.rot_omega);   // src/relax_ic.jl:150-176
        if (A.use_damp) f64::damp_src(d, u0, u1, u2, u3, xc, yc, A.damp_inv_td, A.damp_t, A.damp_omega);
        if (A.mode == 1) {
            // Uin is not written here: other blocks are still staging these
            // cells as halos, and a cell read while its five words were being
            // replaced by their floored values would mix the two states.  The
            // RHS entry points floor Uin in a launch of its own afterwards.
#pragma unroll
            for (int q = 0; q < 5; ++q) A.dU[off + q] = d[q];
            continue;
        }
        double un[5], w[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) un[q] = A.Un[off + q];
        const double uu[5] = {u0, u1, u2, u3, u4};
        if (A.stage == 1) {
#pragma unroll
            for (int q = 0; q < 5; ++q) w[q] = un[q] + dt * d[q];
        } else if (A.stage == 2) {
#pragma unroll
            for (int q = 0; q < 5; ++q) w[q] = 0.75 * un[q] + 0.25 * uu[q] + cdt * d[q];
        } else {
#pragma unroll
            for (int q = 0; q < 5; ++q) w[q] = (1.0 / 3.0) * un[q] + (2.0 / 3.0) * uu[q] + cdt * d[q];
        }
        const double w0 = w[0];
        P::floor(w, A);
        if (LED && A.ledger && led_counted(A, a, b, c)) {
            if (w[0] != w0) atomicAdd(&sled[f64::LED_POST], w[0] - w0);
            if (A.stage > 1) {   // the input's floors reach the combine in stages 2 and 3
                const double raw = A.Uin[off];
                if (u0 != raw) atomicAdd(&sled[f64::LED_PRE], u0 - raw);
            }
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) A.Uout[off + q] = w[q];
        if (A.cfl_max) {
            double s = f64::cfl_speed(w[0], w[1], w[2], w[3], w[4], A.g, A.gm1, A.idx, A.idy, A.idz);
            if (s != s) nanflag = 1;
            else smax = fmax(smax, s);
        }
    }
    if (A.cfl_max) {
        for (int o = 16; o > 0; o >>= 1) smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
        if ((tid & 31) == 0) red[tid >> 5] = smax;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < NT / 32; ++w) m = fmax(m, red[w]);
            atomicMax(A.cfl_max, (unsigned long long)__double_as_longlong(m));
            if (nanflag) atomicOr(A.cfl_nan, 1u);
        }
    }
    if (LED && A.ledger) {
        __syncthreads();   // every cell's and face's contribution is in sled
        if (tid < f64::LED_TERMS && sled[tid] != 0.0) atomicAdd(&A.ledger[tid], sled[tid] * (A.dx * A.dy * A.dz));
    }
    return true;
}

// One launch per stage on one grid: CTA (x, y, z) owns block (x, y, z).
// LED: the instantiation that keeps the mass ledger (A.ledger) -- the driver
// loops' launches; the others compile no ledger code.
template <class P, int TX, int TY, int TZ, int NT, int MINB, bool LED = false>
__global__ void __launch_bounds__(NT, MINB) stage_kernel(const __grid_constant__ f64::StageArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[NT / 32];
    __shared__ unsigned int nanflag;
    if (A.done_dev && *A.done_dev) return;   // device time loop already reached t_end
    P::prologue(policy_smem<P, TX, TY, TZ>(smem_raw), A, NT);   // visible after the first barrier
    stage_block<P, TX, TY, TZ, NT, MINB, LED>(A, blockIdx.x * TX, blockIdx.y * TY, blockIdx.z * TZ, smem_raw, red,
                                              nanflag);
}

// stage_kernel with the cross region staged by TMA copies (tma.cuh): one
// block per CTA, as stage_kernel.  Launched only where build_maps accepted
// the grid (uniform grid, tile dividing it, even nx, no ghost buffer).
template <class P, int TX, int TY, int TZ, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    stage_kernel_tma(const __grid_constant__ f64::StageArgs A, const __grid_constant__ tma::Maps M) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red[NT / 32];
    __shared__ unsigned int nanflag;
    __shared__ __align__(8) uint64_t bar[2];
    if (A.done_dev && *A.done_dev) return;
    using TS = TmaSmem<P, TX, TY, TZ, NT, MINB>;
    using C = typename TS::C;
    P::prologue(policy_smem<P, TX, TY, TZ>(smem_raw), A, NT);
    if (threadIdx.x == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    unsigned char* face = smem_raw + TS::FACE_OFF;
    unsigned char* app = smem_raw + TS::APPEND_OFF;
    TmaCtx T;
    T.M = &M;
    T.raw[0] = reinterpret_cast<double*>(TS::IN_FACES >= 1 ? face : app);
    T.raw[1] = reinterpret_cast<double*>(TS::IN_FACES == 2 ? face + C::RAWB
                                                             : (TS::IN_FACES == 1 ? app : app + C::RAWB));
    T.bar = bar;
    T.ph[0] = T.ph[1] = 0u;
    stage_block<P, TX, TY, TZ, NT, MINB>(A, blockIdx.x * TX, blockIdx.y * TY, blockIdx.z * TZ, smem_raw, red, nanflag,
                                         &T);
}

// The listed blocks of a split stage (written by its screening launch, which
// runs first on the same stream), walked by a persistent grid: each CTA takes
// its first block by its index, then draws the next from a queue counter
// (split_count[1], zeroed with the count), so CTAs whose blocks hold more
// network rows take fewer blocks.
template <class P, int TX, int TY, int TZ, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) stage_kernel_list(const __grid_constant__ f64::StageArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[NT / 32];
    __shared__ unsigned int nanflag;
    __shared__ int next;
    if (A.done_dev && *A.done_dev) return;
    const int n = (int)*A.split_count;
    if ((int)blockIdx.x >= n) return;
    P::prologue(policy_smem<P, TX, TY, TZ>(smem_raw), A, NT);   // visible after the first barrier
    const int gx = (A.nx + TX - 1) / TX, gy = (A.ny + TY - 1) / TY;
    for (int t = blockIdx.x; t < n;) {
        const int b = A.split_list[t];
        stage_block<P, TX, TY, TZ, NT>(A, (b % gx) * TX, ((b / gx) % gy) * TY, (b / (gx * gy)) * TZ, smem_raw, red,
                                       nanflag);
        // the block's barriers order every thread's reads of `next` before this write
        if (threadIdx.x == 0) next = (int)gridDim.x + (int)atomicAdd(A.split_count + 1, 1u);
        __syncthreads();
        t = next;
    }
}

// Several grids (mesh levels or patches of any size) in one launch: their
// blocks form one list, level l owning entries [start[l], start[l+1]); a
// persistent grid of CTAs (as many as fit at once) walks the list, drawing
// blocks from an atomic queue when one is given.  Each level keeps its own
// arguments (states, dt, flux registers, boundary capture), so every block
// computes exactly what its level's own launch would.
template <class P, int TX, int TY, int TZ, int NT, int MINB, bool LED = false>
__global__ void __launch_bounds__(NT, MINB) stage_kernel_batch(const __grid_constant__ f64::StageBatch B) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[NT / 32];
    __shared__ unsigned int nanflag;
    if (B.lv[0].done_dev && *B.lv[0].done_dev) return;
    P::prologue(policy_smem<P, TX, TY, TZ>(smem_raw), B.lv[0], NT);
    const int total = B.start[B.nlev];
    __shared__ int next;
    for (int t = blockIdx.x;; t += gridDim.x) {
        if (B.queue) {   // draw the next block; read by all before any thread draws again
            if (threadIdx.x == 0) next = (int)atomicAdd(B.queue, 1u);
            __syncthreads();
            t = next;
        }
        if (t >= total) break;
        int l = 0;
        while (l + 1 < B.nlev && t >= B.start[l + 1]) ++l;
        const f64::StageArgs& A = B.lv[l];
        const int r = t - B.start[l], gx = B.gx[l], gy = B.gy[l];
        stage_block<P, TX, TY, TZ, NT, MINB, LED>(A, (r % gx) * TX, ((r / gx) % gy) * TY, (r / (gx * gy)) * TZ,
                                                  smem_raw, red, nanflag);
    }
}

template <class P, int TX, int TY, int TZ>
constexpr int smem_bytes() {
    using S = Shape<TX, TY, TZ>;
    return (P::kCols * (P::kCross ? S::NCROSS : S::NEXT) + 5 * S::NFACE) * (int)sizeof(typename P::real) + 16;
}

// Host: launch stage_kernel_batch for the levels in B with a persistent grid
// (at most as many CTAs as fit on the device at once).
template <class P, int TX, int TY, int TZ, int NT, int MINB, bool LED>
bsn_status launch_batch_led(bsn_ctx* ctx, f64::StageBatch B, int smem, const char* name) {
    auto fn = stage_kernel_batch<P, TX, TY, TZ, NT, MINB, LED>;
    static int occ[64] = {0}, sms[64] = {0};
    const int dev = ctx->device & 63;
    if (!occ[dev]) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return cuda_check(ctx, e, "cudaFuncSetAttribute(stage_kernel_batch)");
        int o = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fn, NT, smem);
        if (e != cudaSuccess) return cuda_check(ctx, e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        e = cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, ctx->device);
        if (e != cudaSuccess) return cuda_check(ctx, e, "cudaDeviceGetAttribute");
        occ[dev] = o < 1 ? 1 : o;
    }
    if (B.nlev < 1 || B.nlev > f64::MAXLEV) return set_err(ctx, BSN_ERR_ARG, "batch of %d levels", B.nlev);
    long long total = 0;
    for (int l = 0; l < B.nlev; ++l) {
        const f64::StageArgs& A = B.lv[l];
        long long gx = (A.nx + TX - 1) / TX, gy = (A.ny + TY - 1) / TY, gz = (A.nz + TZ - 1) / TZ;
        B.gx[l] = (int)gx;
        B.gy[l] = (int)gy;
        B.start[l] = (int)total;
        total += gx * gy * gz;
    }
    if (total > 0x7fffffffLL) return set_err(ctx, BSN_ERR_UNSUPPORTED, "too many blocks in one batch");
    B.start[B.nlev] = (int)total;
    long long grid = std::min<long long>(total, (long long)occ[dev] * sms[dev]);
    prof_begin(ctx);
    fn<<<(unsigned)grid, NT, smem, ctx->stream>>>(B);
    return launch_check(ctx, name);
}

// the ledger instantiation when any level keeps a mass ledger
template <class P, int TX, int TY, int TZ, int NT, int MINB>
bsn_status launch_batch(bsn_ctx* ctx, const f64::StageBatch& B, int smem, const char* name) {
    bool led = false;
    for (int l = 0; l < B.nlev && l < f64::MAXLEV; ++l) led = led || B.lv[l].ledger;
    return led ? launch_batch_led<P, TX, TY, TZ, NT, MINB, true>(ctx, B, smem, name)
               : launch_batch_led<P, TX, TY, TZ, NT, MINB, false>(ctx, B, smem, name);
}

// Host: one stage on one grid through stage_kernel (the ledger
// instantiation when A keeps a mass ledger); smem is the dynamic smem.
template <class P, int TX, int TY, int TZ, int NT, int MINB, bool LED>
bsn_status launch_plain_led(bsn_ctx* ctx, const f64::StageArgs& A, int smem, const char* name) {
    auto fn = stage_kernel<P, TX, TY, TZ, NT, MINB, LED>;
    static bool attr_done[64] = {false};
    const int dev = ctx->device & 63;
    if (!attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return cuda_check(ctx, e, "cudaFuncSetAttribute(stage_kernel)");
        attr_done[dev] = true;
    }
    dim3 grid((A.nx + TX - 1) / TX, (A.ny + TY - 1) / TY, (A.nz + TZ - 1) / TZ);
    prof_begin(ctx);
    fn<<<grid, NT, smem, ctx->stream>>>(A);
    return launch_check(ctx, name);
}
template <class P, int TX, int TY, int TZ, int NT, int MINB>
bsn_status launch_plain(bsn_ctx* ctx, const f64::StageArgs& A, int smem, const char* name) {
    return A.ledger ? launch_plain_led<P, TX, TY, TZ, NT, MINB, true>(ctx, A, smem, name)
                    : launch_plain_led<P, TX, TY, TZ, NT, MINB, false>(ctx, A, smem, name);
}

// Host: one stage on one grid through stage_kernel_tma when the grid
// qualifies (tma::build_maps); *used tells whether it was launched.
template <class P, int TX, int TY, int TZ, int NT, int MINB>
bsn_status launch_tma(bsn_ctx* ctx, const f64::StageArgs& A, const char* name, bool* used) {
    using TS = TmaSmem<P, TX, TY, TZ, NT, MINB>;
    using C = typename TS::C;
    *used = false;
    if constexpr (!TS::OK) return BSN_OK;
    if (A.ledger) return BSN_OK;   // the TMA kernel keeps no mass ledger
    tma::Maps M;
    if (!tma::build_maps(ctx, A, TX, TY, TZ, C::AY, C::AZ, C::YZ, C::ZY, M)) return BSN_OK;
    auto fn = stage_kernel_tma<P, TX, TY, TZ, NT, MINB>;
    static bool attr_done[64] = {false};
    const int dev = ctx->device & 63;
    if (!attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, TS::BYTES);
        if (e != cudaSuccess) return cuda_check(ctx, e, "cudaFuncSetAttribute(stage_kernel_tma)");
        attr_done[dev] = true;
    }
    dim3 grid(A.nx / TX, A.ny / TY, A.nz / TZ);
    prof_begin(ctx);
    fn<<<grid, NT, TS::BYTES, ctx->stream>>>(A, M);
    *used = true;
    ctx->tma_used_last = 1;
    return launch_check(ctx, name);
}

}  // namespace tile
}  // namespace bsn
