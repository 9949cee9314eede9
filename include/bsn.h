/*
 * bsn.h -- C ABI of libbsn, the B200 (sm_100a) finite-volume library for
 * Binary-Supernova's hot path.
 *
 * Every entry point replaces one function of the reference Julia package
 * (macfadyen/Binary-Supernova); the citation beside each declaration names
 * the function it stands in for (file:line in the reference).  Arguments keep
 * the reference's meaning and order; Julia keyword arguments become trailing
 * positional arguments.
 *
 * Memory and layout
 *   - Pointers named U, dU, Fx, Fy, Fz, rho, phi are DEVICE pointers owned by
 *     the caller (e.g. `pointer(::CuArray)` from Julia, `tensor.data_ptr()`
 *     from torch).  The library never frees caller memory.
 *   - State arrays use the reference layout U[q,i,j,k] (Julia column-major,
 *     5 conserved variables fastest, NG = 3 ghost cells per side):
 *         U[q + 5*(i + NXT*(j + NYT*k))],  NXT = nx+6, NYT = ny+6, NZT = nz+6,
 *     q = 0..4 = (rho, rho vx, rho vy, rho vz, E), i,j,k 0-based ghosted.
 *     Flux arrays: Fx (5, NXT+1, NYT, NZT), Fy (5, NXT, NYT+1, NZT),
 *     Fz (5, NXT, NYT, NZT+1).  Potentials and densities without ghosts:
 *     phi[i + nx*(j + ny*k)].
 *   - bsn_bh arrays are HOST memory (the reference passes BH data by value).
 *
 * Execution
 *   - Work is ordered on the context's stream.  Functions that return host
 *     values (dt, forces, accretion) synchronise that stream.
 *   - One context per host thread; contexts share nothing.
 *
 * Errors: every call returns bsn_status; bsn_last_error(ctx) gives a message.
 */
#ifndef BSN_H
#define BSN_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int bsn_status;
enum {
    BSN_OK = 0,
    BSN_ERR_ARG = 1,        /* invalid argument (sizes, null pointers, ranges) */
    BSN_ERR_CUDA = 2,       /* a CUDA runtime/driver call failed */
    BSN_ERR_TIMEOUT = 3,    /* a bounded device-side wait expired */
    BSN_ERR_NONFINITE = 4,  /* a NaN/Inf was detected where the reference would throw */
    BSN_ERR_UNSUPPORTED = 5,/* size/feature outside what this build supports */
    BSN_ERR_NOMEM = 6,      /* workspace allocation failed */
    BSN_ERR_IO = 7          /* a checkpoint / snapshot file could not be written or read */
};

enum { BSN_BC_OUTFLOW = 0, BSN_BC_PERIODIC = 1 };

typedef struct bsn_ctx bsn_ctx;

/* Mirrors the reference's mutable BlackHole (src/BinarySupernova.jl:130-137).
 * r_sink/t_sink are derived exactly as src/BinarySupernova.jl:159-171. */
typedef struct {
    double pos[3];
    double vel[3];
    double mass;
    double eps;
    double c_code;
    double r_floor;
} bsn_bh;

/* Two-level FMR grid (src/fmr3d.jl:109-122, FMRGrid3D).  Uc/Uf are device
 * arrays in the state layout; index bounds are the reference's 1-based coarse
 * active-cell indices of the fine patch. */
typedef struct {
    double* Uc; int ncx, ncy, ncz; double dxc, dyc, dzc;
    double* Uf; int nfx, nfy, nfz; double dxf, dyf, dzf;
    int ratio;
    int ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi;
    double gamma;
    int bc;
    double rho_floor, P_floor;
} bsn_fmr2;

/* ---- context (replaces KA.get_backend(U) dispatch, src/gpu_kernels.jl:1-21) */
bsn_status  bsn_ctx_create(bsn_ctx** out, int device, void* cuda_stream);
bsn_status  bsn_ctx_destroy(bsn_ctx* ctx);
bsn_status  bsn_ctx_set_stream(bsn_ctx* ctx, void* cuda_stream);
bsn_status  bsn_ctx_synchronize(bsn_ctx* ctx);
const char* bsn_last_error(const bsn_ctx* ctx);
const char* bsn_version(void);
/* Kernels launched by this context since creation (device launches only). */
long long   bsn_ctx_launch_count(const bsn_ctx* ctx);
/* Per-kernel CUDA-event timing on the context stream.  The reference has no
 * tracing beyond wall-clock progress logs (scripts/run_sn50_fiducial.jl:890-893);
 * these two calls are the library's own instrumentation.  Enabling or
 * disabling clears the records; stats sum every recorded launch of `name`. */
bsn_status  bsn_ctx_set_profiling(bsn_ctx* ctx, int on);
bsn_status  bsn_ctx_kernel_stats(bsn_ctx* ctx, const char* name, double* total_ms, long long* count);
/* Measured multiply-add throughput of the context's GPU in TFLOP/s (one FMA =
 * 2 flops): precision 0 FP64, 1 FP32, 2 FP32 packed (f32x2 FMA).  The
 * denominators of the stencil kernels' FP-pipe fraction; synchronises. */
bsn_status  bsn_fp_peak(bsn_ctx* ctx, int precision, double* tflops);

/* ---- src/euler3d.jl ------------------------------------------------------ */
/* fill_ghost_3d_outflow! / fill_ghost_3d_periodic! (src/euler3d.jl:33-62) */
bsn_status bsn_fill_ghost_3d_f64(bsn_ctx* ctx, double* U, int nx, int ny, int nz, int bc);
/* apply_floors_3d! (src/euler3d.jl:73-80; kernel src/gpu_kernels.jl:26-46) */
bsn_status bsn_apply_floors_3d_f64(bsn_ctx* ctx, double* U, int nx, int ny, int nz,
                                   double rho_floor, double P_floor, double gamma);
/* euler3d_rhs! (src/euler3d.jl:182-205).  Mutates U (ghost fill when
 * fill_ghosts != 0, floors on active cells), fills Fx/Fy/Fz (zero off the
 * interfaces) and dU (zero ghosts).  Fx, Fy, Fz may be NULL to skip them. */
bsn_status bsn_euler3d_rhs_f64(bsn_ctx* ctx, double* dU, double* Fx, double* Fy, double* Fz,
                               double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                               double gamma, int bc, double rho_floor, double P_floor,
                               int fill_ghosts);
/* euler3d_step! (src/euler3d.jl:220-260): one SSP-RK3 step in place. */
bsn_status bsn_euler3d_step_f64(bsn_ctx* ctx, double* U, int nx, int ny, int nz,
                                double dx, double dy, double dz, double dt, double gamma,
                                int bc, double rho_floor, double P_floor);
/* cfl_dt_3d (src/euler3d.jl:157-169; kernel src/gpu_kernels.jl:174-191). */
bsn_status bsn_cfl_dt_3d_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz,
                             double dx, double dy, double dz, double gamma, double cfl,
                             double* dt_out);
/* No counterpart in the reference: the same dt as bsn_cfl_dt_3d_f64, for
 * callers that must not allocate GPU memory (a host runtime that owns a fixed
 * device-memory pool, or a job that sizes all its memory at start-up).  Its
 * scratch is a file-scope static device array of 512 KiB held on every GPU
 * that loads the library until exit; grids above 512^3 = 134,217,728 active
 * cells are rejected with BSN_ERR_UNSUPPORTED.  Under CUDA's lazy module
 * loading the driver reserves the array on a device at the first call there:
 * make one warm-up call at start-up, before a pool takes the device's memory
 * (or set CUDA_MODULE_LOADING=EAGER).  The first call on a device looks up
 * the array's address with that device current; this first call should come
 * before any stream capture.  The context's device must be current
 * (BSN_ERR_ARG otherwise).  All calls share the array: calls that overlap on
 * the GPU race.  The success path allocates nothing. */
bsn_status bsn_cfl_dt_3d_f64_noalloc(bsn_ctx* ctx, const double* U, int nx, int ny, int nz,
                                     double dx, double dy, double dz, double gamma, double cfl,
                                     double* dt_out);

/* ---- fast path and device time loop (no single counterpart in the reference:
 * they run the reference's driver loop, test/test_sedov.jl:45-52 /
 * scripts/run_production.jl:132-135, `dt = cfl_dt_3d; dt = min(dt, t_end-t);
 * euler3d_step!; t += dt`) ---------------------------------------------- */
enum { BSN_PREC_F64 = 0,     /* stencils in FP64, bit-identical to the reference */
       BSN_PREC_F32 = 1,     /* stencils, fluxes and pressures in FP32; state, floors,
                                divergence, sources and RK3 accumulation in FP64 */
       BSN_PREC_LEARNED = 2  /* as BSN_PREC_F32, with the WENO-Z weights of smooth
                                stencils from the learned network (see below) */ };
/* FP32 stencils meet near-vacuum cells beside dense gas (a sink's
 * surroundings, a floor atmosphere): where a face's six-cell density stencil
 * spans more than three decades, FP32 rounding of the dense side's values is
 * 1e-4 and more of the thin cell's, and its velocity m / rho can run away
 * (seen beside the sinks, where the drain empties cells next to dense gas).
 * Such faces are computed in FP64 by the FP64 path's arithmetic in the
 * coupled driver loops with sinks (uniform and nested, bsn_coupled_step_f64)
 * always; the other FP32 loops and steps (bsn_euler3d_step_f32,
 * bsn_run_steps, the FMR and relaxation loops) do it when on != 0 here
 * (default off: a star's surface in a floor atmosphere is a shell of stiff
 * faces, which doubles the FP32 polytrope FMR step).  Releases the context's
 * captured time-loop graphs. */
bsn_status bsn_ctx_set_stiff_guard(bsn_ctx* ctx, int on);
/* euler3d_rhs! with FP32 stencils (BSN_PREC_F32): the same semantics as
 * bsn_euler3d_rhs_f64 (mutates U: ghost fill, floors; fills the optional
 * Fx/Fy/Fz and dU), the face fluxes from the FP32 reconstruction and HLLC
 * (or, with the stiff guard, in FP64 where the density stencil spans more than
 * three decades), stored as FP32 values, the divergence in FP64. */
bsn_status bsn_euler3d_rhs_f32(bsn_ctx* ctx, double* dU, double* Fx, double* Fy, double* Fz, double* U,
                               int nx, int ny, int nz, double dx, double dy, double dz, double gamma, int bc,
                               double rho_floor, double P_floor, int fill_ghosts);
/* euler3d_step! with FP32 stencils (BSN_PREC_F32); same arguments. */
bsn_status bsn_euler3d_step_f32(bsn_ctx* ctx, double* U, int nx, int ny, int nz,
                                double dx, double dy, double dz, double dt, double gamma,
                                int bc, double rho_floor, double P_floor);
/* euler3d_step! with the learned WENO weights (BSN_PREC_LEARNED); needs
 * bsn_learned_set_params first. */
bsn_status bsn_euler3d_step_learned(bsn_ctx* ctx, double* U, int nx, int ny, int nz,
                                    double dx, double dy, double dz, double dt, double gamma,
                                    int bc, double rho_floor, double P_floor);
/* Up to n_steps CFL-limited SSP-RK3 steps with dt, t and the CFL maximum kept
 * on the device (one CUDA graph per step).  t_end > 0 stops at t_end exactly
 * as the reference loop; t_end <= 0 runs n_steps.  *t_inout: start time in,
 * final time out; *steps_done (may be NULL): steps taken.  A dt of 0 (an
 * infinite signal speed) stops the loop with BSN_ERR_NONFINITE. */
bsn_status bsn_run_steps(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double dx, double dy,
                         double dz, double gamma, double cfl, int bc, double rho_floor,
                         double P_floor, int precision, int n_steps, double t_end,
                         double* t_inout, int* steps_done);
/* Tile shape of the fused stage kernel: the library's autotuner times every
 * variant on the first stage of each grid and keeps the fastest, one choice
 * per grid and driver loop (single stages, the uniform, coupled, nested,
 * FMR and relaxation loops); a device loop's first call re-times its tiles
 * after its first step (results are the same with every tile).
 * bsn_ctx_set_tile forces variant `variant` (-1: autotune again);
 * bsn_ctx_get_tile reports the latest choice for a grid as {tx, ty, tz,
 * threads, minimum CTAs per SM the kernel's registers are capped for}. */
/* Staging of the fused stage kernel's block and halos by TMA tensor copies
 * (cp.async.bulk.tensor into shared memory; possible where the tile divides
 * the grid, nx is even and no ghost buffer is involved) beside the plain
 * per-thread loader.  With on != 0 (the default) the autotuner times both
 * stagings of every tile variant and keeps the faster, and a forced variant
 * (bsn_ctx_set_tile) uses TMA wherever possible; on = 0 keeps the plain
 * loader.  Results are the same either way; the switch releases the
 * context's captured step graphs.  bsn_ctx_get_tma reports the setting,
 * bsn_ctx_get_tile_tma whether a grid's chosen tile is TMA-staged (1), not
 * (0) or not chosen yet (-1).  A staging copy that does not arrive within the
 * kernel's wait bound sets an error word, reported as BSN_ERR_TIMEOUT by the
 * next bsn_ctx_synchronize or device time loop. */
bsn_status bsn_ctx_set_tma(bsn_ctx* ctx, int on);
int        bsn_ctx_get_tma(const bsn_ctx* ctx);
int        bsn_ctx_get_tile_tma(bsn_ctx* ctx, int precision, int nx, int ny, int nz);
int        bsn_tile_variant_count(int precision);
bsn_status bsn_ctx_set_tile(bsn_ctx* ctx, int precision, int variant);
bsn_status bsn_ctx_get_tile(bsn_ctx* ctx, int precision, int nx, int ny, int nz, int out[5]);

/* ---- learned WENO weights (no counterpart in the reference; plain WENO5-Z of
 * src/weno5.jl:14-61 is its yardstick).  Two networks, for the left- and the
 * right-biased reconstruction, each 5 -> 32 -> 32 -> 3 (ReLU, softmax), map
 * a normalised 5-point stencil u_i = (v_i - v_c)/max|v_j - v_c| to the three
 * weights.  A reconstruction uses the network only where the smoothness
 * indicators of u say the stencil is smooth (tau5 <= 4 (min beta + 1e-3)) and
 * its spread max|v_j - v_c| exceeds 1e-15 and 1e-6 |v_c| (FP32 rounding
 * level); elsewhere plain WENO5-Z.  Parameters: FP32, bsn_learned_param_count()
 * floats per network, layout W1[32][5] b1[32] W2[32][32] b2[32] W3[3][32] b3[3].
 * All arrays below are device memory. */
int        bsn_learned_param_count(void);
/* Training samples from a state: for every interface and field (rho, m, P),
 * the normalised left/right stencils and their FP64 WENO-Z weights, smooth
 * stencils only, and only those whose spread max|v_i - v_c| exceeds both
 * 1e-15 and 1e-12 |v_c| (below that any weights reconstruct to rounding
 * level), each kept with probability 1/stride.  Samples are 8 floats
 * (u[5], omega[3]) appended at index counts[side]; counts (in: current, out:
 * new) count every kept stencil, the buffers hold the first min(count, cap). */
bsn_status bsn_learned_collect(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, int bc,
                               double gamma, int stride, unsigned long long seed,
                               float* out_left, float* out_right, long long cap, long long counts[2]);
/* Mean-squared-error gradient of one network over all n samples (sum over
 * samples; *loss = summed squared error), by the training kernels. */
bsn_status bsn_learned_grad(bsn_ctx* ctx, const float* samples, long long n, const float* params,
                            float* grad, double* loss);
/* Adam on mini-batches of `batch` samples (multiple of 128) drawn uniformly
 * with replacement, learning rate decayed from lr to 0 on a cosine; params
 * updated in place; *last_loss = mean squared error of the last batch. */
bsn_status bsn_learned_train(bsn_ctx* ctx, const float* samples, long long n, float* params, int steps,
                             int batch, float lr, unsigned long long seed, double* last_loss);
/* Install trained parameters for BSN_PREC_LEARNED (packed to BF16 for the
 * tensor cores; FP32 biases). */
bsn_status bsn_learned_set_params(bsn_ctx* ctx, const float* params_left, const float* params_right);
/* Weights of n normalised stencils u[n][5] -> w[n][3]: tensor_cores = 0 runs
 * the FP32 training arithmetic, 1 the BF16 mma path of the stencil kernel. */
bsn_status bsn_learned_eval(bsn_ctx* ctx, const float* u, long long n, const float* params, float* w,
                            int tensor_cores);

/* ---- src/gravity_bh.jl, src/sinks.jl ------------------------------------ */
/* add_bh_gravity_source! (src/gravity_bh.jl:58-78; src/gpu_kernels.jl:199-230) */
bsn_status bsn_add_bh_gravity_source_f64(bsn_ctx* ctx, double* dU, const double* U,
                                         int nx, int ny, int nz, double dx, double dy, double dz,
                                         const bsn_bh* bhs, int nbh, double x0, double y0, double z0);
/* gas_force_on_bh (src/gravity_bh.jl:91-113) -> out[3] (host). */
bsn_status bsn_gas_force_on_bh_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz,
                                   double dx, double dy, double dz, const bsn_bh* bh,
                                   double x0, double y0, double z0, double out[3]);
/* add_sink_sources! (src/sinks.jl:32-59; src/gpu_kernels.jl:238-284) */
bsn_status bsn_add_sink_sources_f64(bsn_ctx* ctx, double* dU, const double* U,
                                    int nx, int ny, int nz, double dx, double dy, double dz,
                                    const bsn_bh* bhs, int nbh, double x0, double y0, double z0,
                                    double f_sink, int torque_free, double rho_sink_min);
/* accrete! (src/sinks.jl:74-109): mutates *bh (host). */
bsn_status bsn_accrete_f64(bsn_ctx* ctx, bsn_bh* bh, const double* U, int nx, int ny, int nz,
                           double dx, double dy, double dz, double x0, double y0, double z0,
                           double dt, double f_sink, double rho_sink_min);
/* The same sources on a z-slab of a larger grid (one rank's planes of a
 * z-decomposed grid; the reference runs on one device and has no slab form):
 * k0 is the global index of the slab's first active plane, and cell centres
 * are z0 + (k0 + k + 0.5) dz with the global index, so every cell takes the
 * undivided grid's arithmetic bit for bit.  gas_force_on_bh's slab form gives
 * the slab's compensated partial sums as (hi, lo) pairs per component
 * (out[6]); bsn_merge_force_pairs merges the ranks' pairs in rank order (the
 * same two-sum merge as the device reduction) into the force. */
bsn_status bsn_add_bh_gravity_source_slab_f64(bsn_ctx* ctx, double* dU, const double* U,
                                              int nx, int ny, int nz, double dx, double dy, double dz,
                                              const bsn_bh* bhs, int nbh, double x0, double y0, double z0, int k0);
bsn_status bsn_add_sink_sources_slab_f64(bsn_ctx* ctx, double* dU, const double* U,
                                         int nx, int ny, int nz, double dx, double dy, double dz,
                                         const bsn_bh* bhs, int nbh, double x0, double y0, double z0,
                                         double f_sink, int torque_free, double rho_sink_min, int k0);
bsn_status bsn_gas_force_on_bh_slab_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz,
                                        double dx, double dy, double dz, const bsn_bh* bh,
                                        double x0, double y0, double z0, int k0, double out[6]);
bsn_status bsn_merge_force_pairs(const double* pairs, int nparts, double out[3]);
/* One SSP-RK3 stage of euler3d_step! / coupled_step! (src/euler3d.jl:220-260,
 * scripts/run_sn50_fiducial.jl:767-790) as one fused launch, with the input's
 * ghost cells as the caller left them (filled, and on a z-slab exchanged with
 * the neighbouring slabs): Uout = the stage combination of Un and the floored
 * Uin with the right-hand side of Uin plus the sources, then floored.  Uout
 * must differ from Uin; stage 1 takes Un = Uin (the unfloored U^n, as the
 * reference combines).  Sources (src may be NULL): BH gravity of bhs[0..nbh),
 * the sinks of bhs[0..nsink) (src/gpu_kernels.jl:199-284), the self-gravity
 * gradient of phi (nx ny nz, the potential of the stage input's floored
 * density) with the neighbouring slabs' planes phi_lo / phi_hi (NULL at the
 * global boundary); cell centres x0 + (i + 0.5) dx ... with the slab's first
 * global plane k0.  precision: BSN_PREC_*; the FP32 forms compute stiff faces
 * in FP64 when sinks are on (bsn_ctx_set_stiff_guard otherwise).  The ghost
 * cells of Uout: after stage 3 with Uout = Un (the state U, whose ghost cells
 * must then still hold U^n's) the reference's whole-array combination
 * (1/3) U^n + (2/3) Uin there; otherwise left as they were (the next stage's
 * fill replaces them).  Stage 1's input must not be U itself when the caller
 * fills its ghosts (U^n's ghost cells enter that combination).  No single
 * reference counterpart: the reference's stage is euler3d_rhs! plus the
 * source calls plus the combination. */
typedef struct {
    const bsn_bh* bhs; int nbh; int nsink;
    double f_sink; int torque_free; double rho_sink_min;
    double x0, y0, z0; int k0;
    const double* phi; const double* phi_lo; const double* phi_hi;
} bsn_stage_sources;
bsn_status bsn_euler3d_stage(bsn_ctx* ctx, double* Uout, double* Uin, const double* Un, int nx, int ny, int nz,
                             double dx, double dy, double dz, double dt, double gamma, int stage,
                             double rho_floor, double P_floor, int precision, const bsn_stage_sources* src);
/* accrete! (src/sinks.jl:74-109) over slabs, in three parts whose result is
 * the undivided accrete! bit for bit: bsn_sink_box gives the global active
 * box (0-based inclusive {ilo,ihi,jlo,jhi,klo,khi}) that holds the sink
 * sphere on the global nx x ny x nz grid (host); each rank's
 * bsn_sink_terms_slab_f64 writes the terms the reference's sums add for the
 * cells of that box in its planes, in the reference's (k, j, i) order, into
 * the host buffer terms (4 doubles per cell: rho, mx, my, mz times
 * dV / t_sink * dt, zeros outside the sphere or at rho <= rho_sink_min;
 * *count cells, at most cap); the ranks' term lists concatenated in rank
 * order are the global list, and bsn_accrete_from_terms adds them in order
 * and updates the BH (host). */
bsn_status bsn_sink_box(const bsn_bh* bh, int nx, int ny, int nz, double dx, double dy, double dz,
                        double x0, double y0, double z0, int box[6]);
bsn_status bsn_sink_terms_slab_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz,
                                   double dx, double dy, double dz, double x0, double y0, double z0, int k0,
                                   const bsn_bh* bh, double dt, double f_sink, double rho_sink_min,
                                   const int box[6], double* terms, long long cap, long long* count);
bsn_status bsn_accrete_from_terms(bsn_bh* bh, const double* terms, long long n);
/* nbody_step! (src/nbody.jl:74-104), host FP64.  F_gas is nbh*3 host doubles. */
bsn_status bsn_nbody_step(bsn_bh* bhs, int nbh, double dt, const double* F_gas);
/* KeplerOrbit(bhs; com, nhat, Omega) (src/kepler_orbit.jl:63-111), host FP64.
 * nhat may be NULL (inferred), Omega <= 0 means inferred.  state[13] out. */
bsn_status bsn_kepler_init(const bsn_bh* bhs, const double com[3], const double* nhat,
                           double Omega, double state[13]);
/* kepler_update! (src/kepler_orbit.jl:124-150), host FP64. */
bsn_status bsn_kepler_update(bsn_bh* bhs, const double state[13], double t);

/* ---- src/self_gravity.jl, src/fmr_gravity.jl ---------------------------- */
/* solve_poisson_isolated (src/self_gravity.jl:35-76): rho, phi device (nx,ny,nz). */
bsn_status bsn_solve_poisson_isolated_f64(bsn_ctx* ctx, const double* rho, int nx, int ny, int nz,
                                          double dx, double dy, double dz, double* phi);
/* The same solve with FP32 transforms (the precision form of the FFTs): FP64
 * rho in and phi out, FP32 spectra and Green's function. */
bsn_status bsn_solve_poisson_isolated_f32(bsn_ctx* ctx, const double* rho, int nx, int ny, int nz,
                                          double dx, double dy, double dz, double* phi);
/* solve_poisson_isolated of an nx x ny x nz grid split into z-slabs, one per
 * rank (no reference counterpart: the reference solves on one device).  The
 * three calls are the solve cut at its z transform; between them the caller
 * moves data between ranks (an all-to-all), and the assembled potential is
 * bit-identical to bsn_solve_poisson_isolated_f64.  W2, T: interleaved
 * complex doubles, W2[kx + (nx+1)*(ky + 2ny*z)] for the slab's nzl planes,
 * T[kx + (nx+1)*(kyl + nky*z)] for ky = ky0 + kyl and all nz planes; rho, phi
 * (nx, ny, nzl).  nx, ny (and the global nz) powers of two.
 * slab_forward: x, y transforms of the slab's density planes into W2.
 * slab_zconv: z transform, Green's function of the global grid, inverse z
 *   transform of the lines of T, in place.
 * slab_inverse: y, x inverse transforms of W2 into the slab's potential. */
bsn_status bsn_poisson_slab_forward_f64(bsn_ctx* ctx, const double* rho, int nx, int ny, int nzl, double* W2);
bsn_status bsn_poisson_slab_zconv_f64(bsn_ctx* ctx, double* T, int nx, int ny, int nz, int ky0, int nky,
                                      double dx, double dy, double dz);
bsn_status bsn_poisson_slab_inverse_f64(bsn_ctx* ctx, const double* W2, int nx, int ny, int nzl, double* phi);
/* _apply_sg_force_level! (src/fmr_gravity.jl:146-156; src/gpu_kernels.jl:291-319) */
bsn_status bsn_sg_gradient_f64(bsn_ctx* ctx, double* dU, const double* U, const double* phi,
                               int nx, int ny, int nz, double dx, double dy, double dz);
/* _apply_sg_force_level! on a z-slab of a larger grid (src/gpu_kernels.jl:
 * 291-319 applied to the larger grid): phi_lo / phi_hi (device, nx*ny, may be
 * NULL) are the planes of Phi just below / above the slab, so the slab's edge
 * planes take the central z difference of the larger grid's cells; NULL at the
 * larger grid's own boundary keeps the reference's one-sided difference. */
bsn_status bsn_sg_gradient_slab_f64(bsn_ctx* ctx, double* dU, const double* U, const double* phi,
                                    const double* phi_lo, const double* phi_hi, int nx, int ny, int nz,
                                    double dx, double dy, double dz);
/* add_self_gravity_source! (src/self_gravity.jl:93-115) */
bsn_status bsn_add_self_gravity_source_f64(bsn_ctx* ctx, double* dU, const double* U,
                                           int nx, int ny, int nz, double dx, double dy, double dz);

/* ---- src/relax_ic.jl ------------------------------------------------------ */
/* rotating_frame_source! (src/relax_ic.jl:150-176): centrifugal and Coriolis
 * terms of a frame rotating at Omega about z through the origin, added to dU. */
bsn_status bsn_rotating_frame_source_f64(bsn_ctx* ctx, double* dU, const double* U, int nx, int ny, int nz,
                                         double dx, double dy, double dz, double x0, double y0, double z0,
                                         double Omega);
/* relax_damping_source! (src/relax_ic.jl:59-120): velocity damping over t_damp
 * toward the co-rotation velocity (-Omega y, Omega x, 0), added to dU. */
bsn_status bsn_relax_damping_source_f64(bsn_ctx* ctx, double* dU, const double* U, int nx, int ny, int nz,
                                        double dx, double dy, double dz, double x0, double y0, double z0,
                                        double t_damp, double Omega);
/* relax_ic! (src/relax_ic.jl:200-330) on the device: SSP-RK3 with the hydro
 * RHS, BH gravity (bhs, host, held fixed), self-gravity per stage when
 * self_gravity != 0, the rotating frame when Omega != 0 and damping toward
 * rest, until t_max, KE/E_thermal < KE_tol, or the ratio turns back up 10 %
 * past its post-peak minimum; at most max_steps steps.  dt, t and the stop
 * rule stay on the device, one CUDA graph per step.  precision: BSN_PREC_*
 * stencils.  Outputs (may be NULL): final t, steps taken, last KE ratio. */
bsn_status bsn_relax_ic(bsn_ctx* ctx, double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                        double gamma, const bsn_bh* bhs, int nbh, double x0, double y0, double z0,
                        double t_damp, double t_max, double cfl, double rho_floor, double P_floor,
                        double KE_tol, double Omega, int self_gravity, int precision, int max_steps,
                        double* t_out, int* n_steps_out, double* ke_ratio_out);

/* ---- driver stage order: coupled_step! (scripts/run_sn50_fiducial.jl:756-818)
 * BH forces, optional nbody_step! (evolve_orbit), three fused RK3 stages with
 * BH gravity, optional self-gravity and sinks, then accrete!.  bhs is host
 * memory and is updated; Fgas_out (host, nbh*3, may be NULL) receives F_gas. */
bsn_status bsn_coupled_step_f64(bsn_ctx* ctx, double* U, bsn_bh* bhs, int nbh, double dt, double t,
                                int nx, int ny, int nz, double dx, double x0, double y0, double z0,
                                double gamma, double f_sink, double rho_floor, double P_floor,
                                int torque_free, int self_gravity, double t_bh2_sink_on,
                                double rho_sink_min, int evolve_orbit, double* Fgas_out);
/* The driver loop around coupled_step! on the device: up to n_steps steps of
 * dt = min(CFL dt, dt_max if > 0, t_end - t if t_end > 0) then coupled_step!,
 * with the BHs, t and dt in device memory (gas forces, nbody_step!, source
 * parameters and accrete! computed there) and each step one CUDA graph.
 * bhs: host in/out.  precision: BSN_PREC_* stencils (sources, orbits and
 * accretion FP64); FP32 transforms for self-gravity unless BSN_PREC_F64.
 * *t_inout: start time in, final out; *steps_done (may be NULL).  diag_out
 * (device, may be NULL): after every step k < diag_cap the record of
 * BSN_DIAG_RECORD doubles {t, dt, the 10 values of bsn_diagnostics_f64, the
 * mass ledger} at diag_out + BSN_DIAG_RECORD k, reduced on the device (no
 * per-step copy to the host).  The mass ledger, FP64 totals since the start
 * of the call: [12] mass the floors added, [13] mass that left through the
 * domain boundary, [14] mass the sink sources drained from the gas, [15]
 * mass accrete! credited to the BHs; the gas mass [11] closes as
 * M_gas(0) + [12] - [13] - [14].  [15] - [14] is the reference's own
 * difference between accrete! (end-of-step state, src/sinks.jl:74-109) and
 * the stage drain (src/gpu_kernels.jl:238-284). */
enum { BSN_DIAG_RECORD = 16 };
bsn_status bsn_coupled_run_steps(bsn_ctx* ctx, double* U, bsn_bh* bhs, int nbh, int nx, int ny, int nz,
                                 double dx, double x0, double y0, double z0, double gamma, double cfl,
                                 double dt_max, double f_sink, double rho_floor, double P_floor,
                                 int torque_free, int self_gravity, double t_bh2_sink_on,
                                 double rho_sink_min, int evolve_orbit, int precision, int n_steps,
                                 double t_end, double* t_inout, int* steps_done, double* diag_out,
                                 int diag_cap);
/* The same driver loop on nested FMR levels (no counterpart in the reference,
 * whose coupled_step! runs on one uniform grid): per step dt = the nested CFL
 * (bsn_cfl_dt_fmr_nested_f64, capped and clamped as above); the gas force on
 * every BH from the composite of the levels (each level's cells except those
 * its child covers); nbody_step!; one nested step (bsn_fmr_nested_step_f64)
 * whose stages on every level carry BH gravity, self-gravity (Phi frozen per
 * level-0 step, solved on level 0) and sinks in coupled_step!'s order, BHs
 * frozen at their post-orbit state; accrete! from the finest level over dt.
 * pairs: as bsn_fmr_nested_step_f64 (gamma, floors from pairs[0]); x0,y0,z0:
 * lower corner of level 0 (each finer level starts at the lower face of its
 * parent's cell ci_lo).  diag_out records are the diagnostics of level 0,
 * which holds the restriction of the finer levels, with the mass ledger of
 * the composite grid (each level counts the cells its child does not cover;
 * level 0 the domain boundary).  Start from levels that hold the restriction
 * of their children for the ledger to close from the first step. */
bsn_status bsn_coupled_nested_run_steps(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, bsn_bh* bhs, int nbh,
                                        double x0, double y0, double z0, double cfl, double dt_max,
                                        double f_sink, int torque_free, int self_gravity, double t_bh2_sink_on,
                                        double rho_sink_min, int evolve_orbit, int precision, int n_steps,
                                        double t_end, double* t_inout, int* steps_done, double* diag_out,
                                        int diag_cap);
/* The driver's diagnostics (src/diagnostics.jl:21-175) in one device
 * reduction: out[0] gas_energy_total, [1] gas_kinetic_total, [2..4]
 * gas_momentum_total, [5..7] gas_angular_momentum_total, [8]
 * bound_gas_mass(bhs, gamma), [9] the gas mass sum(rho) dV.  Whole-grid sums
 * compensated (within about one rounding of the exact sum).  bhs: host. */
bsn_status bsn_diagnostics_f64(bsn_ctx* ctx, const double* U, int nx, int ny, int nz, double dx,
                               double dy, double dz, double x0, double y0, double z0,
                               const bsn_bh* bhs, int nbh, double gamma, double out[10]);

/* ---- src/fmr3d.jl ----------------------------------------------------------- */
/* FMRGrid3D constructor's _prolong_all! (src/fmr3d.jl:131-151, 206-214) */
bsn_status bsn_fmr_prolong_all_f64(bsn_ctx* ctx, const bsn_fmr2* G);
/* _prolong_fine_ghosts! (src/fmr3d.jl:223-255) from coarse array Uc_src */
bsn_status bsn_fmr_prolong_fine_ghosts_f64(bsn_ctx* ctx, double* Uf, const double* Uc_src,
                                           const bsn_fmr2* G);
/* _restrict! (src/fmr3d.jl:266-285) */
bsn_status bsn_fmr_restrict_f64(bsn_ctx* ctx, double* Uc, const double* Uf, const bsn_fmr2* G);
/* fmr3d_step! (src/fmr3d.jl:451-604) */
bsn_status bsn_fmr3d_step_f64(bsn_ctx* ctx, const bsn_fmr2* G, double dt_c, int self_gravity,
                              double G_grav);
/* cfl_dt_fmr3d (src/fmr3d.jl:616-622) */
bsn_status bsn_cfl_dt_fmr3d_f64(bsn_ctx* ctx, const bsn_fmr2* G, double cfl, double* dt_out);
/* restrict_density_to_coarse! (src/fmr_gravity.jl:40-60) */
bsn_status bsn_restrict_density_to_coarse_f64(bsn_ctx* ctx, const bsn_fmr2* G);
/* solve_fmr_poisson (src/fmr_gravity.jl:119-133): phi_c (ncx,ncy,ncz), phi_f (nfx,nfy,nfz) device */
bsn_status bsn_solve_fmr_poisson_f64(bsn_ctx* ctx, const bsn_fmr2* G, double* phi_c, double* phi_f);
/* _prolong_scalar_trilinear! (src/fmr_gravity.jl:70-106): phi_f (nfx,nfy,nfz)
 * from phi_c (ncx,ncy,ncz), both device, column-major active grids */
bsn_status bsn_prolong_scalar_trilinear_f64(bsn_ctx* ctx, const bsn_fmr2* G, const double* phi_c, double* phi_f);
/* The FMR driver loop `dt = cfl_dt_fmr3d(G, cfl); dt = min(dt, t_end - t);
 * fmr3d_step!(G, dt; self_gravity, G_grav); t += dt` (src/fmr3d.jl:451-622)
 * run on the device: up to n_steps steps, t_end > 0 stops at t_end exactly
 * (t_end <= 0 runs n_steps); dt, t and the CFL maxima stay on the device and
 * each step is one CUDA graph.  The coarse RK3 step and the first fine
 * subcycle are updated together, one persistent launch over the blocks of
 * both levels per RK3 stage; the remaining subcycles follow.  precision:
 * BSN_PREC_F64 (stencils as fmr3d_step), BSN_PREC_F32 or BSN_PREC_LEARNED.
 * The first subcycle takes its ghosts from U_c^n itself where the reference
 * interpolates 1*U_c^n + 0*U_c^{n+1}: results are equal except for the sign
 * of a zero and a non-finite U_c^{n+1}.  *t_inout: start time in, final time
 * out; *steps_done (may be NULL): steps taken. */
bsn_status bsn_fmr3d_run_steps(bsn_ctx* ctx, const bsn_fmr2* G, double cfl, int precision, int self_gravity,
                               double G_grav, int n_steps, double t_end, double* t_inout, int* steps_done);

/* ---- nested FMR, N = npairs + 1 <= 4 levels.  The reference's fmr3d_step!
 * (src/fmr3d.jl:451-604) couples two levels; these entries generalise it
 * recursively: each level subcycles `ratio` times inside its parent's step
 * with ghosts from the parent at a = s/ratio, registers and Berger-Colella
 * correction per pair, self-gravity solved on level 0 and interpolated down
 * the chain (src/fmr_gravity.jl pair by pair).  pairs[k] couples level k
 * (Uc) with level k+1 (Uf); pairs[k].Uf must be pairs[k+1].Uc with matching
 * extents and spacings.  gamma, bc and floors are taken from pairs[0].  At
 * npairs = 1 they equal the two-level entries above. */
bsn_status bsn_fmr_nested_step_f64(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, double dt0, int self_gravity,
                             double G_grav);
/* min over levels l of (ratio_0 ... ratio_{l-1}) * cfl / max signal speed of l */
bsn_status bsn_cfl_dt_fmr_nested_f64(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, double cfl, double* dt_out);
/* The nested driver loop on the device, one CUDA graph per level-0 step (as
 * bsn_fmr3d_run_steps).  The first substeps of a chain of levels l..N-1 take
 * their ghosts from their parents' states at the start of the parents'
 * substeps, so each RK3 stage of such a chain is one persistent launch over
 * all of its levels. */
bsn_status bsn_fmr_nested_run_steps(bsn_ctx* ctx, const bsn_fmr2* pairs, int npairs, double cfl, int precision,
                              int self_gravity, double G_grav, int n_steps, double t_end, double* t_inout,
                              int* steps_done);

/* ---- src/checkpoint.jl, src/io.jl: HDF5 checkpoints, snapshots, trajectories
 * The files are written by the library's own HDF5 writer (no HDF5 library is
 * linked): version-2 superblock and object headers, compact groups,
 * attributes in the object headers, contiguous little-endian float64 / int64
 * datasets, null-terminated ASCII string attributes; array dimensions in
 * HDF5 order, i.e. reversed from the reference's column-major shapes with
 * the same bytes (the way HDF5.jl stores a Julia array).  The readers take
 * the files this library writes.  Group, dataset and attribute names, shapes
 * and meanings are the reference's. */
typedef struct {   /* the /manifest scalars of a uniform checkpoint */
    double t; long long step; double dt_last, t_snap, t_bh2_sink_on;
} bsn_ckpt_meta;
typedef struct {   /* the /grid attributes of a uniform checkpoint */
    int nx, ny, nz; double dx, dy, dz, gamma, x0, y0, z0, rho_floor, P_floor;
} bsn_grid_meta;
/* save_checkpoint_uniform (src/checkpoint.jl:222-265): U the ghosted state
 * (device memory when on_device != 0, else host), bhs host.  Returns when the
 * file is written. */
bsn_status bsn_save_checkpoint_uniform(bsn_ctx* ctx, const char* path, const double* U, int on_device,
                                       const bsn_bh* bhs, int nbh, const bsn_grid_meta* grid,
                                       const bsn_ckpt_meta* meta);
/* The same checkpoint without stopping the run: a device copy of U ordered on
 * the context's stream (work enqueued after the call may change U), then a
 * copy to pinned host memory on a copy stream and the file write on a host
 * thread.  bsn_checkpoint_wait joins it and returns its status; a second
 * asynchronous checkpoint on the context first waits for the previous one. */
bsn_status bsn_save_checkpoint_uniform_async(bsn_ctx* ctx, const char* path, const double* U_dev,
                                             const bsn_bh* bhs, int nbh, const bsn_grid_meta* grid,
                                             const bsn_ckpt_meta* meta);
bsn_status bsn_checkpoint_wait(bsn_ctx* ctx);
/* load_checkpoint_uniform (src/checkpoint.jl:277-318).  With U = NULL only
 * grid, meta and *nbh are read (to size the arrays); then U (device or host,
 * 5 (nx+6)(ny+6)(nz+6) doubles) and bhs (room for cap_bh) are filled.  Rejects
 * a checkpoint whose format_version is not 1 or whose kind is not "uniform". */
bsn_status bsn_load_checkpoint_uniform(bsn_ctx* ctx, const char* path, double* U, int on_device, bsn_bh* bhs,
                                       int cap_bh, int* nbh, bsn_grid_meta* grid, bsn_ckpt_meta* meta);
/* save_checkpoint / load_checkpoint of a two-level FMR grid
 * (src/checkpoint.jl:39-165): G's level arrays on the device (on_device != 0)
 * or host.  load fills G's geometry, gamma, bc and floors from the file; with
 * G->Uc / G->Uf non-NULL it also reads the level states into them (the fine
 * level as saved, not re-prolonged). */
bsn_status bsn_save_checkpoint_fmr(bsn_ctx* ctx, const char* path, const bsn_fmr2* G, int on_device,
                                   const bsn_bh* bhs, int nbh, double t, long long step, double dt_last);
bsn_status bsn_load_checkpoint_fmr(bsn_ctx* ctx, const char* path, bsn_fmr2* G, int on_device, bsn_bh* bhs,
                                   int cap_bh, int* nbh, double* t, long long* step, double* dt_last);
/* write_snapshot / read_snapshot (src/io.jl:29-83): /gas/{rho,rhovx,rhovy,
 * rhovz,E} of the active cells and root attributes t, nx, ny, nz, dx, dy, dz,
 * gamma.  read_snapshot fills U_active[q, i, j, k] (5 nx ny nz doubles, host;
 * NULL to read the attributes only). */
bsn_status bsn_write_snapshot(bsn_ctx* ctx, const char* path, const double* U, int on_device, int nx, int ny,
                              int nz, double dx, double dy, double dz, double t, double gamma);
bsn_status bsn_read_snapshot(const char* path, double* U_active, long long cap, int* nx, int* ny, int* nz,
                             double* dx, double* dy, double* dz, double* t, double* gamma);
/* init_trajectory_file / append_trajectory / read_trajectory (src/io.jl:96-
 * 180): /time and /bh{i}/{mass, rsink, pos, vel}; the reference extends
 * chunked datasets, here each append rewrites the file one record longer.
 * read fills t[N], mass/rsink[b*N + r], pos/vel[(b*N + r)*3 + d] (room for
 * cap dumps; t = NULL reads the counts only). */
bsn_status bsn_trajectory_init(const char* path, int n_bh);
bsn_status bsn_trajectory_append(const char* path, double t, const bsn_bh* bhs, int nbh);
bsn_status bsn_trajectory_read(const char* path, int* n_dumps, int* n_bh, double* t, double* mass, double* pos,
                               double* vel, double* rsink, long long cap);

#ifdef __cplusplus
}
#endif
#endif /* BSN_H */
