// fmr_nested.cuh -- the nested-level FMR step plan (fmr_nlevel.cu), shared
// with the coupled driver loop on nested levels (coupled_run.cu).
#pragma once

#include "fmr.cuh"

namespace bsn {
namespace fmr {

constexpr int NMAXL = f64::MAXLEV;   // levels
constexpr int NMAXQ = 64;            // batched stage launches per coarse step

struct NDev {
    double dt[NMAXL];                // substep dt of each level
    double t;
    unsigned long long sm[NMAXL];    // CFL maxima (double bits)
    unsigned int nan[NMAXL];
    int done, steps;
    unsigned int queue[NMAXQ];       // block queues of the batched launches (zeroed every step)
};

struct Ratios {
    int r[NMAXL];
    int n;                           // levels
};

struct NLevel {
    double *U, *Ucn, *A, *B, *Gh, *phi;
    int nx, ny, nz;
    double dx, dy, dz;
};

struct NPair {
    Geo G;
    Regs Rc, Rf;
    double* regs;                    // Rc and Rf, contiguous
    long long nregs;                 // doubles in regs
    long long nfine;                 // threads of fine_reg_kernel
    long long ncorr;                 // threads of bc_correct_kernel
};

// Device buffers of all levels and pairs in one allocation, laid out from the
// level sizes (the same sizes give the same pointers, so a captured graph
// stays valid).
struct NArena {
    void* base = nullptr;
    size_t bytes = 0;
};

struct NState {
    NArena arena;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
    std::vector<bsn_fmr2> key_pairs;
    int prec = -1, sg = 0;
    double G_grav = 0, cfl = 0, t_end = 0;
    int tiles[NMAXL] = {-1, -1, -1, -1};
    void* key_base = nullptr;
    std::vector<double> key_extra;   // further parameters of the captured step (coupled loop)
    cudaStream_t cap = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
};

struct NPlan {
    bsn_ctx* ctx = nullptr;
    int nl = 0, prec = PREC_F64, sg = 0;
    double G_grav = 1.0;
    NLevel L[NMAXL];
    NPair P[NMAXL - 1];
    f64::StageArgs base[NMAXL];
    Ratios R;
    NDev* d = nullptr;
    const int* done = nullptr;
    int qn = 0;
    double rho_floor = 0, P_floor = 0, gamma = 0;
    int bc = 0;
    // optional mass ledger of the composite grid: per level the per-stage
    // sums of the substep being taken (3 x LED_TERMS doubles, device), and
    // the cumulative totals (LEDT_COUNT doubles, device).  Each level counts
    // its cells outside its child's region; level 0 also its boundary faces.
    double* led_raw[NMAXL] = {nullptr, nullptr, nullptr, nullptr};
    double* led_tot = nullptr;

    LedBox covered(int l) const;    // level l's cells that level l+1 covers (none for the finest)
    bsn_status chain(int l, double alpha);
    bsn_status gravity();
    bsn_status step();
};

// Validate a chain of level pairs (pairs[k].Uf == pairs[k+1].Uc), lay out the
// device buffers of all levels in S's arena and fill the plan: stage
// arguments per level (registers toward the child, boundary faces toward the
// parent, ghosts from the parent, Phi with self-gravity, dt read on the
// device).  Callers may add sources to plan.base[l] before plan.step().
bsn_status make_plan(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, int prec, int sg, double G_grav, int guard, NState* S,
                     NPlan& plan);

// graphs, stream, events and arena of a state, then the state itself
void nstate_destroy(NState* S);

__global__ void n_init_kernel(NDev* d, double t);
__global__ void n_fixed_dt_kernel(NDev* d, double dt0, Ratios R);
__global__ void n_dt_kernel(NDev* d, double cfl, Ratios R, double t_end, double dt_max);
__global__ void n_advance_kernel(NDev* d);

}  // namespace fmr
}  // namespace bsn
