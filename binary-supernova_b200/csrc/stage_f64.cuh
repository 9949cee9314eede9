// stage_f64.cuh -- arguments of the fused RK3-stage kernel (stage_tile.cuh)
// and its FP64 tile constants.  Fluxes never go to HBM unless the caller asks
// for them (euler3d_rhs!) or a flux register needs them (FMR).
#pragma once

#include "physics.cuh"

namespace bsn {
namespace f64 {

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
    double fac;              // weight * dt (host dt)
    double wt;               // weight, used with a device-resident dt
};
// Fine-level boundary faces captured for ordered register accumulation.
struct BndFaces {
    double* f[6];            // xlo,xhi,ylo,yhi,zlo,zhi, each (5, na, nb) over active transverse
};

struct StageArgs {
    double* Uin;             // stage input (stencil source); floored after the launch in RHS mode
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
    const double* dt_dev;    // non-null: dt read on the device (graph-captured time loop)
    const int* done_dev;     // non-null and *done_dev != 0: the device time loop has finished
    const void* mlp;         // learned stencil path: packed network parameters
    // learned stage split in two launches: the screening launch (plain FP32
    // stencils) does every block whose three sweeps are uniform and lists the
    // others here; the learned launch then does the listed blocks
    int learned_split;            // learned stages split (uniform-grid entry points; off elsewhere)
    int* split_list;              // block index bx + gx (by + gy bz)
    unsigned int* split_count;
    const BHSrc* bh_dev;     // non-null: gravity sources read on the device (device-resident driver loop)
    const SinkSrc* sk_dev;   // non-null: sink sources read on the device
    // relaxation sources (src/relax_ic.jl): rotating frame at rot_omega,
    // velocity damping over damp_t (damp_inv_td = 1 / damp_t) toward rotation at damp_omega
    int use_rot, use_damp;
    double rot_omega, damp_t, damp_inv_td, damp_omega;
    // mass ledger (null: off).  Four sums of rho dV for this stage, added
    // with atomics: [LED_BND] mass flux into the grid through its own
    // boundary faces per unit time (counted when led_bnd != 0, i.e. the grid's
    // boundary is the domain's), [LED_DRAIN] the sink drain rho / t_sink per
    // unit time, [LED_POST] the change made by the floors after the combine,
    // [LED_PRE] the change the floors made to the stage input where the
    // combine uses it (stages 2 and 3).  Cells in [led_skip_lo, led_skip_hi)
    // (a finer level's region, overwritten by its restriction) are not counted.
    double* ledger;
    int led_bnd;
    int led_skip_lo[3], led_skip_hi[3];
    // FP32 path: compute faces whose density stencil spans more than three
    // decades in FP64 (the F32Guarded policy)
    int stiff_guard;
    // the grid as a z-slab of a larger one: global index of its first active
    // plane (cell centres of the sources), and the planes of Phi just below /
    // above it (null at the larger grid's boundary) for the self-gravity
    // gradient at the slab's edge planes
    int k0;
    const double* phi_lo;
    const double* phi_hi;
    // the driver loop this stage belongs to (TUNE_* in stage_launch.cuh): the
    // autotuner keeps one tile choice per driver and grid, so a driver's
    // choice is timed on its own stage arguments and grid contents
    int tune_class;
};

enum { LED_BND = 0, LED_DRAIN = 1, LED_POST = 2, LED_PRE = 3, LED_TERMS = 4 };
// cumulative mass-ledger totals of a driver loop (rho dV): mass added by the
// floors, mass that left through the domain boundary, mass the sink sources
// drained from the gas, mass the sinks' accrete! credited to the BHs
enum { LEDT_FLOORS = 0, LEDT_OUTFLOW = 1, LEDT_DRAINED = 2, LEDT_ACCRETED = 3, LEDT_COUNT = 4 };

// Centre of active cell (a, b, c) (0-based): x0 + (i - ng - 0.5) dx with
// i = a + 1 + ng (src/gravity_bh.jl:63-65).
__device__ __forceinline__ void cell_xyz(int a, int b, int c, double x0, double y0, double z0, double dx, double dy,
                                         double dz, double& xc, double& yc, double& zc) {
    xc = x0 + ((double)(a + 1) - 0.5) * dx;
    yc = y0 + ((double)(b + 1) - 0.5) * dy;
    zc = z0 + ((double)(c + 1) - 0.5) * dz;
}

// Several grids (mesh levels, patches of any size) updated by one launch:
// level l's blocks are entries [start[l], start[l+1]) of one block list,
// gx/gy its blocks along x and y (filled by the launcher from the tile).
// queue: a zeroed counter the CTAs draw blocks from (dynamic schedule);
// null: CTA b takes blocks b, b + gridDim, ...
constexpr int MAXLEV = 4;
struct StageBatch {
    StageArgs lv[MAXLEV];
    unsigned int* queue;
    int nlev;
    int gx[MAXLEV], gy[MAXLEV];
    int start[MAXLEV + 1];
};



}  // namespace f64
}  // namespace bsn
