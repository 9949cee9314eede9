// stage_f64.cuh -- the fused FP64 RK3-stage kernel.
//
// One CTA owns an 8x8x8 block of active cells.  For each sweep direction it
// stages the block plus a 3-cell halo along that direction in shared memory
// (floors applied to active cells, ghost cells taken raw from the boundary
// map or a ghost buffer), computes every interface flux of the block once
// (WENO5-Z + HLLC), and accumulates the flux divergence of its cells in
// registers.  The epilogue adds the source terms in the reference's order
// (BH gravity, self-gravity, sinks), applies the SSP-RK3 combine and the
// floors, stores the stage result and optionally folds the next CFL speed
// into a device-wide max.  Fluxes never go to HBM unless the caller asks for
// them (euler3d_rhs!) or a flux register needs them (FMR).
#pragma once

#include "physics.cuh"

namespace bsn {
namespace f64 {

constexpr int TX = 8, TY = 8, TZ = 8;
constexpr int NT = 256;
constexpr int NCELL = TX * TY * TZ;
constexpr int CPT = NCELL / NT;
constexpr int NEXT = (TX + 6) * TY * TZ;     // cells of one direction-extended block
constexpr int NFACE = (TX + 1) * TY * TZ;    // interfaces of one direction
constexpr int SMEM_BYTES = (6 * NEXT + 5 * NFACE) * 8 + 64;
static_assert(TX == TY && TY == TZ, "extended-block sizes assume a cubic tile");

constexpr int MAXBH = 4;

struct BHSrc {       // gravity sources (src/gpu_kernels.jl:199-230)
    int n;
    double px[MAXBH], py[MAXBH], pz[MAXBH], mass[MAXBH], eps[MAXBH];
};
struct SinkSrc {     // sink sources (src/gpu_kernels.jl:238-284)
    int n, torque_free;
    double rho_min;
    double px[MAXBH], py[MAXBH], pz[MAXBH], vx[MAXBH], vy[MAXBH], vz[MAXBH], rs[MAXBH], ts[MAXBH];
};

// Coarse-level Berger-Colella register faces (src/fmr3d.jl:292-326).
// Face indices are 0-based active-relative "left face of cell a" positions.
struct RegFaces {
    double* reg[6];          // xlo,xhi,ylo,yhi,zlo,zhi, each (5, t1, t2)
    int lo[3], hi[3];        // face positions along x,y,z (lo = ci_lo-1, hi = ci_hi)
    int t0[3], t1[3];        // transverse active ranges [t0, t1] per axis
    double fac;              // weight * dt
};
// Fine-level boundary faces captured for ordered register accumulation.
struct BndFaces {
    double* f[6];            // xlo,xhi,ylo,yhi,zlo,zhi, each (5, na, nb) over active transverse
};

struct StageArgs {
    double* Uin;             // stage input (stencil source); written back in RHS mode
    const double* Gh;        // ghost source array (same layout); null -> boundary map of Uin
    const double* Un;        // combine base (stage mode)
    double* Uout;            // stage result (stage mode)
    double* dU;              // RHS result (RHS mode)
    double* F[3];            // optional interface materialisation (reference shapes)
    int nx, ny, nz, bc;
    int mode;                // 0 = RK3 stage, 1 = euler3d_rhs!
    int stage;               // 1, 2, 3
    double g, gm1, rho_floor, P_floor, Pfl_gm1;
    double idx, idy, idz;
    double dt, cdt;          // cdt = 0.25*dt (stage 2), (2/3)*dt (stage 3)
    // sources
    int use_bh, use_sink, use_sg;
    double x0, y0, z0, dx, dy, dz;
    BHSrc bh;
    SinkSrc sk;
    const double* phi;       // (nx,ny,nz) active grid
    double inv2dx, inv2dy, inv2dz;
    int use_reg, use_bnd;
    RegFaces reg;
    BndFaces bnd;
    unsigned long long* cfl_max;   // non-null: fold CFL speed of the output
    unsigned int* cfl_nan;
};

#ifdef BSN_DEFINE_STAGE_KERNEL
__device__ __forceinline__ void load_cell(const StageArgs& A, const Geom& G, int d, int a, int b, int c,
                                          double v[5], bool& active) {
    // (a,b,c) active-relative; only coordinate d may lie in the ghost band.
    int n[3] = {G.nx, G.ny, G.nz};
    int p[3] = {a, b, c};
#pragma unroll
    for (int t = 0; t < 3; ++t)
        if (t != d) p[t] = p[t] < n[t] ? p[t] : n[t] - 1;   // partial tile: clamp (unused)
    int pd = p[d];
    active = (pd >= 0 && pd < n[d]);
    long long off;
    const double* src;
    if (active) {
        src = A.Uin;
        off = G.act(p[0], p[1], p[2]);
    } else if (A.Gh) {
        pd = pd < -BSN_NG ? -BSN_NG : (pd > n[d] + BSN_NG - 1 ? n[d] + BSN_NG - 1 : pd);
        p[d] = pd;
        src = A.Gh;
        off = G.act(p[0], p[1], p[2]);
    } else {
        p[d] = bc_map(pd, n[d], A.bc);
        src = A.Uin;
        off = G.act(p[0], p[1], p[2]);
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) v[q] = src[off + q];
}

template <int D>
__device__ void sweep(const StageArgs& A, const Geom& G, int a0, int b0, int c0, double* sC, double* sF,
                      double (&acc)[CPT][5]) {
    constexpr int LX = TX + (D == 0 ? 6 : 0), LY = TY + (D == 1 ? 6 : 0);
    constexpr int FX = TX + (D == 0), FY = TY + (D == 1);
    const int tid = threadIdx.x;
    const int n[3] = {G.nx, G.ny, G.nz};
    const int o[3] = {a0, b0, c0};

    __syncthreads();
    // ---- stage the direction-extended block (SoA: var-major in smem)
    for (int e = tid; e < NEXT; e += NT) {
        int ex = e % LX, r = e / LX, ey = r % LY, ez = r / LY;
        int a = a0 + ex - (D == 0 ? 3 : 0);
        int b = b0 + ey - (D == 1 ? 3 : 0);
        int c = c0 + ez - (D == 2 ? 3 : 0);
        double v[5];
        bool act;
        load_cell(A, G, D, a, b, c, v, act);
        if (act) apply_floor(v[0], v[1], v[2], v[3], v[4], A.rho_floor, A.P_floor, A.Pfl_gm1, A.gm1);
#pragma unroll
        for (int q = 0; q < 5; ++q) sC[q * NEXT + e] = v[q];
        sC[5 * NEXT + e] = cell_pressure(v[0], v[1], v[2], v[3], v[4], A.gm1);
    }
    __syncthreads();

    // ---- every interface of the block along D
    constexpr int SD = (D == 0) ? 1 : (D == 1 ? LX : LX * LY);   // smem stride along D
    for (int f = tid; f < NFACE; f += NT) {
        int fx = f % FX, r = f / FX, fy = r % FY, fz = r / FY;
        int fpos[3] = {fx, fy, fz};
        // global face position along D and transverse coordinates
        bool valid = true;
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            int gpos = o[t] + fpos[t];
            valid = valid && (t == D ? gpos <= n[t] : gpos < n[t]);
        }
        if (!valid) continue;
        int base = fx + LX * (fy + LY * fz);   // extended index of stencil cell 0
        double c[6][6];
#pragma unroll
        for (int s = 0; s < 6; ++s)
#pragma unroll
            for (int q = 0; q < 6; ++q) c[s][q] = sC[q * NEXT + base + s * SD];
        double F[5];
        interface_flux<D>(c, A.g, A.gm1, F);
#pragma unroll
        for (int q = 0; q < 5; ++q) sF[q * NFACE + f] = F[q];

        // ownership of the shared block-boundary face: the tile whose first
        // cell it bounds, or the last tile for the domain's last face
        int gd = o[D] + fpos[D];
        bool owner = (fpos[D] < (D == 0 ? TX : (D == 1 ? TY : TZ))) || (gd == n[D]);
        if (!owner) continue;
        int ga = o[0] + fx, gb = o[1] + fy, gc = o[2] + fz;
        if (A.F[D]) {
            // reference array index: face "left of active cell g" -> ghosted
            // interface index g + NG - 1 along D
            long long ex_ = (G.nx + 2 * BSN_NG) + (D == 0), ey_ = (G.ny + 2 * BSN_NG) + (D == 1);
            long long ii = ga + BSN_NG - (D == 0), jj = gb + BSN_NG - (D == 1), kk = gc + BSN_NG - (D == 2);
            long long off = 5LL * (ii + ex_ * (jj + ey_ * kk));
#pragma unroll
            for (int q = 0; q < 5; ++q) A.F[D][off + q] = F[q];
        }
        if (A.use_reg) {
            const RegFaces& R = A.reg;
            int ta = (D == 0) ? gb : ga, tb = (D == 2) ? gb : gc;   // transverse (t1, t2) coords
            int ax1 = (D == 0) ? 1 : 0, ax2 = (D == 2) ? 1 : 2;
            if (ta >= R.t0[ax1] && ta <= R.t1[ax1] && tb >= R.t0[ax2] && tb <= R.t1[ax2]) {
                int n1 = R.t1[ax1] - R.t0[ax1] + 1;
                long long roff = 5LL * ((ta - R.t0[ax1]) + (long long)n1 * (tb - R.t0[ax2]));
                double* dst = nullptr;
                if (gd == R.lo[D]) dst = R.reg[2 * D];
                else if (gd == R.hi[D]) dst = R.reg[2 * D + 1];
                if (dst) {
#pragma unroll
                    for (int q = 0; q < 5; ++q) dst[roff + q] += R.fac * F[q];
                }
            }
        }
        if (A.use_bnd && (gd == 0 || gd == n[D])) {
            int ta = (D == 0) ? gb : ga, tb = (D == 2) ? gb : gc;
            int n1 = (D == 0) ? G.ny : G.nx;
            long long roff = 5LL * (ta + (long long)n1 * tb);
            double* dst = A.bnd.f[2 * D + (gd == 0 ? 0 : 1)];
#pragma unroll
            for (int q = 0; q < 5; ++q) dst[roff + q] = F[q];
        }
    }
    __syncthreads();

    // ---- divergence contribution of this direction for owned cells
    const double inv = (D == 0) ? A.idx : (D == 1 ? A.idy : A.idz);
    constexpr int FS = (D == 0) ? 1 : (D == 1 ? FX : FX * FY);   // face stride along D
#pragma unroll
    for (int m = 0; m < CPT; ++m) {
        int cell = tid + m * NT;
        int i = cell % TX, j = (cell / TX) % TY, k = cell / (TX * TY);
        int fl = i + FX * (j + FY * k);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            double dF = sF[q * NFACE + fl + FS] - sF[q * NFACE + fl];
            if (D == 0) acc[m][q] = -dF * inv;
            else acc[m][q] = acc[m][q] - dF * inv;
        }
    }
}

__global__ void __launch_bounds__(NT, 2) stage_kernel(StageArgs A) {
    extern __shared__ __align__(16) double smem[];
    double* sC = smem;
    double* sF = smem + 6 * NEXT;
    __shared__ double red[NT / 32];
    __shared__ unsigned int nanflag;

    Geom G(A.nx, A.ny, A.nz);
    const int a0 = blockIdx.x * TX, b0 = blockIdx.y * TY, c0 = blockIdx.z * TZ;
    const int tid = threadIdx.x;
    if (tid == 0) nanflag = 0;

    double acc[CPT][5];
    sweep<0>(A, G, a0, b0, c0, sC, sF, acc);
    sweep<1>(A, G, a0, b0, c0, sC, sF, acc);
    sweep<2>(A, G, a0, b0, c0, sC, sF, acc);

    // ---- epilogue: the z-extended block still holds the floored stage input
    double smax = 0.0;
#pragma unroll
    for (int m = 0; m < CPT; ++m) {
        int cell = tid + m * NT;
        int i = cell % TX, j = (cell / TX) % TY, k = cell / (TX * TY);
        int a = a0 + i, b = b0 + j, c = c0 + k;
        if (a >= A.nx || b >= A.ny || c >= A.nz) continue;
        int e = i + TX * (j + TY * (k + 3));
        double u0 = sC[0 * NEXT + e], u1 = sC[1 * NEXT + e], u2 = sC[2 * NEXT + e], u3 = sC[3 * NEXT + e],
               u4 = sC[4 * NEXT + e];
        double* d = acc[m];
        double xc = A.x0 + ((double)(a + 1) - 0.5) * A.dx;
        double yc = A.y0 + ((double)(b + 1) - 0.5) * A.dy;
        double zc = A.z0 + ((double)(c + 1) - 0.5) * A.dz;
        if (A.use_bh) {   // src/gpu_kernels.jl:199-230
            double vx = u1 / u0, vy = u2 / u0, vz = u3 / u0;
            double ax = 0.0, ay = 0.0, az = 0.0;
            for (int nb = 0; nb < A.bh.n; ++nb) {
                double ddx = xc - A.bh.px[nb], ddy = yc - A.bh.py[nb], ddz = zc - A.bh.pz[nb];
                double r2 = sq(ddx) + sq(ddy) + sq(ddz) + sq(A.bh.eps[nb]);
                double r3 = r2 * sqrt(r2);
                double fac = -A.bh.mass[nb] / r3;
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
            const double* P = A.phi;
            long long sy = nx, sz = (long long)nx * ny;
            double gx = (P[ip + sy * b + sz * c] - P[im + sy * b + sz * c]) * fx;
            double gy = (P[a + sy * jp + sz * c] - P[a + sy * jm + sz * c]) * fy;
            double gz = (P[a + sy * b + sz * kp] - P[a + sy * b + sz * km]) * fz;
            double vdotg = (u1 * gx + u2 * gy + u3 * gz) / u0;
            d[1] -= u0 * gx; d[2] -= u0 * gy; d[3] -= u0 * gz; d[4] -= u0 * vdotg;
        }
        if (A.use_sink && u0 > A.sk.rho_min) {   // src/gpu_kernels.jl:238-284
            for (int nb = 0; nb < A.sk.n; ++nb) {
                double ddx = xc - A.sk.px[nb], ddy = yc - A.sk.py[nb], ddz = zc - A.sk.pz[nb];
                double rr = sqrt(sq(ddx) + sq(ddy) + sq(ddz));
                if (rr < A.sk.rs[nb]) {
                    double ts = A.sk.ts[nb];
                    d[0] -= u0 / ts;
                    if (A.sk.torque_free) {
                        double rx = ddx / rr, ry = ddy / rr, rz = ddz / rr;
                        double vx = u1 / u0, vy = u2 / u0, vz = u3 / u0;
                        double vrx = vx - A.sk.vx[nb], vry = vy - A.sk.vy[nb], vrz = vz - A.sk.vz[nb];
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
        long long off = G.act(a, b, c);
        if (A.mode == 1) {
#pragma unroll
            for (int q = 0; q < 5; ++q) A.dU[off + q] = d[q];
            A.Uin[off + 0] = u0; A.Uin[off + 1] = u1; A.Uin[off + 2] = u2; A.Uin[off + 3] = u3;
            A.Uin[off + 4] = u4;
            continue;
        }
        double un[5], w[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) un[q] = A.Un[off + q];
        const double uu[5] = {u0, u1, u2, u3, u4};
        if (A.stage == 1) {
#pragma unroll
            for (int q = 0; q < 5; ++q) w[q] = un[q] + A.dt * d[q];
        } else if (A.stage == 2) {
#pragma unroll
            for (int q = 0; q < 5; ++q) w[q] = 0.75 * un[q] + 0.25 * uu[q] + A.cdt * d[q];
        } else {
#pragma unroll
            for (int q = 0; q < 5; ++q) w[q] = (1.0 / 3.0) * un[q] + (2.0 / 3.0) * uu[q] + A.cdt * d[q];
        }
        apply_floor(w[0], w[1], w[2], w[3], w[4], A.rho_floor, A.P_floor, A.Pfl_gm1, A.gm1);
#pragma unroll
        for (int q = 0; q < 5; ++q) A.Uout[off + q] = w[q];
        if (A.cfl_max) {
            double s = cfl_speed(w[0], w[1], w[2], w[3], w[4], A.g, A.gm1, A.idx, A.idy, A.idz);
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
            // non-negative doubles order like their bit patterns
            atomicMax(A.cfl_max, (unsigned long long)__double_as_longlong(m));
            if (nanflag) atomicOr(A.cfl_nan, 1u);
        }
    }
}

#endif  // BSN_DEFINE_STAGE_KERNEL

}  // namespace f64
}  // namespace bsn
