// fmr.cuh -- fixed mesh refinement operators shared by the two-level path
// (fmr_f64.cu) and the nested N-level path (fmr_nlevel.cu): level-pair
// geometry, prolongation, restriction, flux registers and the
// Berger-Colella correction of src/fmr3d.jl, src/fmr_gravity.jl.
#pragma once

#include "stage_launch.cuh"
#include "hydro_f64.cuh"

namespace bsn {
namespace fmr {

constexpr int MAXR = 8;

struct Geo {
    int ncx, ncy, ncz, nfx, nfy, nfz, r;
    int lo[3], hi[3];        // 1-based coarse active index range of the patch
    double w[MAXR * 5];      // Lagrange-5 weights, w[s + r*j] (src/fmr3d.jl:32-46)
};

struct Regs {
    double* r[6];           // xlo, xhi, ylo, yhi, zlo, zhi: (5, t1, t2) coarse
    const double* bnd[6];
};
// Validates a level pair and fills its geometry and Lagrange-5 weights.
bsn_status make_geo(bsn_ctx* ctx, const bsn_fmr2* g, Geo& G);
long long ghost_count(int nx, int ny, int nz);

__global__ void prolong_ghosts_kernel(Geo G, const double* Ucn, const double* Ucnp1, double alpha, double* dst,
                                      const int* done);
__global__ void restrict_kernel(Geo G, double* Uc, const double* Uf, int qmax, const int* done);
__global__ void fine_reg_kernel(Geo G, Regs R, double fac, const double* dtf_dev, double wt, double rr,
                                const int* done);
__global__ void bc_correct_kernel(Geo G, Regs Rc, Regs Rf, double* Uc, double idx, double idy, double idz,
                                  const int* done);
__global__ void trilinear_kernel(Geo G, const double* pc, double* pf);
__global__ void scale_kernel(double* a, long long n, double s);
__global__ void copy_kernel(double* dst, const double* src, long long n, const int* done);
__global__ void zero_kernel(double* a, long long n, const int* done);

// Fine ghost cells from (1 - alpha) Ucn + alpha Ucnp1 (Ucnp1 null: Ucn).
bsn_status prolong_ghosts(bsn_ctx* ctx, const Geo& G, const double* Ucn, const double* Ucnp1, double alpha,
                          double* dst, const int* done = nullptr);
// qmax = 5: _restrict!; qmax = 1: restrict_density_to_coarse!
bsn_status restrict_(bsn_ctx* ctx, const Geo& G, double* Uc, const double* Uf, int qmax, const int* done = nullptr);
bsn_status fmr_poisson(bsn_ctx* ctx, const bsn_fmr2* g, const Geo& G, double* phic, double* phif, bool fp32 = false);

}  // namespace fmr
}  // namespace bsn
