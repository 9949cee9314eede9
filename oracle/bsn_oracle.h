/*
 * bsn_oracle.h -- CPU FP64 oracle for the Binary-Supernova finite-volume path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference leg
 * may load it.  The product (libbsn, the CUDA path) never links or calls it.
 *
 * It is a line-by-line restatement in C++ of the reference's Julia code
 * (macfadyen/Binary-Supernova, src/ *.jl), FP64, no FMA contraction, exact
 * Julia evaluation order (a+b+c == (a+b)+c, a*b*c == (a*b)*c, x^2 == x*x).
 *
 * Parity pins: the reference ships no golden vectors and Julia is not present,
 * so this oracle is pinned by the reference's own known-answer tests
 * (test/test_weno5.jl, test_sod3d.jl, test_sedov.jl, test_fmr3d.jl,
 * test_sinks.jl, test_self_gravity.jl, test_fmr_gravity.jl, test_nbody.jl,
 * test_kepler_orbit.jl, test_blackhole.jl) and by the accuracy figures the
 * reference documents (docs/phase1.md, phase2.md, phase7.md).
 *
 * Array layout: Julia column-major U[q,i,j,k], q fastest, 0-based flat index
 * q + 5*(i + NXT*(j + NYT*k)), NXT = nx+6 etc.  Flux arrays Fx have shape
 * (5, NXT+1, NYT, NZT), Fy (5, NXT, NYT+1, NZT), Fz (5, NXT, NYT, NZT+1).
 */
#ifndef BSN_ORACLE_H
#define BSN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors the reference's mutable BlackHole (src/BinarySupernova.jl:130-137). */
typedef struct {
    double pos[3];
    double vel[3];
    double mass;
    double eps;
    double c_code;
    double r_floor;
} orc_bh;

/* Two-level FMR grid (src/fmr3d.jl:109-122).  Index bounds are the reference's
 * 1-based coarse active-cell indices.  Uc/Uf are caller-owned ghosted arrays. */
typedef struct {
    double *Uc; int ncx, ncy, ncz; double dxc, dyc, dzc;
    double *Uf; int nfx, nfy, nfz; double dxf, dyf, dzf;
    int ratio;
    int ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi;
    double gamma;
    int bc;               /* 0 outflow, 1 periodic */
    double rho_floor, P_floor;
} orc_fmr;

/* weno5.jl */
double orc_weno5_left(double vm2, double vm1, double v0, double vp1, double vp2);
double orc_weno5_right(double vm1, double v0, double vp1, double vp2, double vp3);
void   orc_wenoz_weights(double b0, double b1, double b2, double d0, double d1, double d2, double out[3]);
/* hllc.jl: dir 0=x,1=y,2=z; L[5], R[5] = (rho,mx,my,mz,E) */
void   orc_hllc_flux(int dir, const double* L, const double* R, double gamma, double out[5]);

/* euler3d.jl */
void   orc_set_threads(int n);
void   orc_fill_ghost_outflow(double* U, int nx, int ny, int nz);
void   orc_fill_ghost_periodic(double* U, int nx, int ny, int nz);
void   orc_apply_floors(double* U, int nx, int ny, int nz, double rho_floor, double P_floor, double gamma);
void   orc_weno_fluxes(int dir, double* F, const double* U, int nx, int ny, int nz, double gamma);
void   orc_flux_divergence(double* dU, const double* Fx, const double* Fy, const double* Fz,
                           int nx, int ny, int nz, double dx, double dy, double dz);
double orc_cfl_dt_3d(const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                     double gamma, double cfl);
void   orc_euler3d_rhs(double* dU, double* Fx, double* Fy, double* Fz, double* U,
                       int nx, int ny, int nz, double dx, double dy, double dz, double gamma,
                       int bc, double rho_floor, double P_floor, int fill_ghosts);
void   orc_euler3d_step(double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                        double dt, double gamma, int bc, double rho_floor, double P_floor);
void   orc_sedov_ic_3d(double* U, int nx, int ny, int nz, double dx, double dy, double dz, double gamma,
                       double E_blast, double r_inject, double rho_bg, double P_floor,
                       double x_offset, double y_offset, double z_offset);

/* BinarySupernova.jl, gravity_bh.jl, sinks.jl, nbody.jl, kepler_orbit.jl */
double orc_r_sink(const orc_bh* bh);
double orc_t_sink(const orc_bh* bh, double f_sink);
void   orc_add_bh_gravity_source(double* dU, const double* U, int nx, int ny, int nz,
                                 double dx, double dy, double dz, const orc_bh* bhs, int nbh,
                                 double x0, double y0, double z0);
void   orc_gas_force_on_bh(const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                           const orc_bh* bh, double x0, double y0, double z0, double out[3]);
void   orc_add_sink_sources(double* dU, const double* U, int nx, int ny, int nz,
                            double dx, double dy, double dz, const orc_bh* bhs, int nbh,
                            double x0, double y0, double z0, double f_sink, int torque_free,
                            double rho_sink_min);
void   orc_add_bh_gravity_source_slab(double* dU, const double* U, int nx, int ny, int nz,
                                      double dx, double dy, double dz, const orc_bh* bhs, int nbh,
                                      double x0, double y0, double z0, int kofs);
void   orc_gas_force_on_bh_slab(const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                                const orc_bh* bh, double x0, double y0, double z0, int kofs, double out[3]);
void   orc_add_sink_sources_slab(double* dU, const double* U, int nx, int ny, int nz,
                                 double dx, double dy, double dz, const orc_bh* bhs, int nbh,
                                 double x0, double y0, double z0, double f_sink, int torque_free,
                                 double rho_sink_min, int kofs);
long   orc_sink_terms_slab(const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                           double x0, double y0, double z0, int kofs, const orc_bh* bh, double rate,
                           double rho_sink_min, int ilo, int ihi, int jlo, int jhi, int klo, int khi,
                           double* out);
void   orc_accrete(orc_bh* bh, const double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                   double x0, double y0, double z0, double dt, double f_sink, double rho_sink_min);
void   orc_nbody_step(orc_bh* bhs, int nbh, double dt, const double* F_gas /* [nbh][3] */);
/* KeplerOrbit: state[0..2]=com, [3]=Omega, [4..6]=nhat, [7..12]=r_init[2][3] */
int    orc_kepler_init(const orc_bh* bhs, const double com[3], const double* nhat_or_null,
                       double Omega_or_nonpositive, double state[13]);
void   orc_kepler_update(orc_bh* bhs, const double state[13], double t);

/* self_gravity.jl, fmr_gravity.jl */
void   orc_fft3d(double* re, double* im, int n1, int n2, int n3, int inverse);
void   orc_solve_poisson_isolated(const double* rho, int nx, int ny, int nz,
                                  double dx, double dy, double dz, double* phi);
void   orc_sg_gradient(double* dU, const double* U, const double* phi, int nx, int ny, int nz,
                       double dx, double dy, double dz);
void   orc_add_self_gravity_source(double* dU, const double* U, int nx, int ny, int nz,
                                   double dx, double dy, double dz);

/* driver stage order (scripts/run_sn50_fiducial.jl:756-818).  Un, dU, Fx, Fy,
 * Fz are scratch of the usual shapes.  Returns F_gas in Fgas_out[nbh*3]. */
void   orc_coupled_step(double* U, double* Un, double* dU, double* Fx, double* Fy, double* Fz,
                        orc_bh* bhs, int nbh, double dt, double t, int nx, int ny, int nz,
                        double dx, double x0, double y0, double z0, double gamma,
                        double f_sink, double rho_floor, double P_floor, int torque_free,
                        int self_gravity, double t_bh2_sink_on, double rho_sink_min,
                        int evolve_orbit, double* Fgas_out);

/* fmr3d.jl */
void   orc_lag5_weights(int ratio, double* w /* ratio x 5, column-major like Julia */);
void   orc_prolong_all(const orc_fmr* G);
void   orc_prolong_fine_ghosts(double* Uf, const double* Uc, const orc_fmr* G);
void   orc_restrict(double* Uc, const double* Uf, const orc_fmr* G);
void   orc_fmr3d_step(const orc_fmr* G, double dt_c, int self_gravity, double G_grav);
double orc_cfl_dt_fmr3d(const orc_fmr* G, double cfl);
/* relax_ic.jl */
void   orc_rotating_frame_source(double* dU, const double* U, int nx, int ny, int nz, double dx, double dy,
                                 double dz, double x0, double y0, double z0, double Om);
void   orc_relax_damping_source(double* dU, const double* U, int nx, int ny, int nz, double dx, double dy,
                                double dz, double x0, double y0, double z0, double t_damp, double Om);
void   orc_relax_ic(double* U, int nx, int ny, int nz, double dx, double dy, double dz, double g,
                    const orc_bh* bhs, int nbh, double x0, double y0, double z0, double t_damp, double t_max,
                    double cfl, double rho_floor, double P_floor, double KE_tol, double Om, int self_gravity,
                    int max_steps, double out[3]);
/* N nested levels: pairs[k].Uf is pairs[k+1].Uc */
void   orc_fmrN_step(const orc_fmr* pairs, int npairs, double dt0, int self_gravity, double G_grav);
double orc_cfl_dt_fmrN(const orc_fmr* pairs, int npairs, double cfl);
/* gas_force_on_bh over the composite of nested levels (level 0 origin x0,y0,z0) */
void   orc_gas_force_fmrN(const orc_fmr* pairs, int npairs, const orc_bh* bh, double x0, double y0, double z0,
                          double out[3]);
/* coupled_step! on nested levels: composite gas force, orbit, nested step
 * with BH gravity / self-gravity / sinks on every level, accretion on the
 * finest level */
void   orc_coupled_fmrN_step(const orc_fmr* pairs, int npairs, orc_bh* bhs, int nbh, double dt0, double t,
                             double x0, double y0, double z0, double f_sink, int torque_free, int self_gravity,
                             double t_bh2_sink_on, double rho_sink_min, int evolve_orbit, double* Fgas);
void   orc_restrict_density_to_coarse(const orc_fmr* G);
void   orc_prolong_scalar_trilinear(double* phi_f, const double* phi_c, const orc_fmr* G);
void   orc_solve_fmr_poisson(const orc_fmr* G, double* phi_c, double* phi_f);

/* stellar_ic.jl (input generators) */
int    orc_lane_emden(double n, double dxi, double* xi_1, double* dtheta_1, double* thetas, int cap);
void   orc_polytrope_ic_3d(double* U, int nx, int ny, int nz, double dx, double dy, double dz, double gamma,
                           double M_star, double R_star, double M_core, double x0, double y0, double z0,
                           double xc, double yc, double zc, double rho_floor, double P_floor,
                           double out[4]);
double orc_thermal_bomb(double* U, int nx, int ny, int nz, double dx, double dy, double dz,
                        double E_SN, double r_bomb, double r_bomb_inner, double x0, double y0, double z0,
                        double xc, double yc, double zc, double bipolar_theta_deg);

#ifdef __cplusplus
}
#endif
#endif
