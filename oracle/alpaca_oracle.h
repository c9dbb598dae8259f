/* TEST INFRASTRUCTURE ONLY — the CPU oracle, never part of the product path.
 *
 * A plain-C restatement of ALPACA's per-block finite-volume right-hand side and
 * SSP-RK3 stage update (the reference is tumaer/ALPACA, files cited per function
 * in alpaca_oracle.c). Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * arm call it, as the checker of the CUDA path.
 *
 * Layout = the reference's Block buffers (block_definitions/field_buffer.h:37-40):
 * per block and field a C-ordered double[TCX][TCY][TCZ] with TC = 24 in every
 * active dimension and 1 in inactive ones (z fastest). Conservatives are ordered
 * Mass, Energy, MomentumX[, MomentumY[, MomentumZ]] (field_setup.h:101-131),
 * prime states Density, Pressure, VelocityX[, VelocityY[, VelocityZ]].
 * Face fluxes use the reference's [NE][ICX+1][ICY+1][ICZ+1] arrays
 * (convective_term_solver.h:67-81), IC = 16 in active and 1 in inactive dims.
 */
#ifndef ALPACA_ORACLE_H
#define ALPACA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Scheme selectors, the same enum values as the reference's
 * user_specifications (riemann_solver_settings.h:29-31,
 * state_reconstruction_settings.h:27). */
enum { ORACLE_FLUX_SPLITTING = 0, ORACLE_FINITE_VOLUME = 1 };
enum { ORACLE_RECON_CONSERVATIVE = 0, ORACLE_RECON_PRIMITIVE = 1,
       ORACLE_RECON_CHARACTERISTIC = 2 };

int oracle_weno5(const double *v6, double *left, double *right);

/* Selects the reconstruction stencil, Riemann solver, signal speed and flux
 * splitting for the calls that follow (values of the reference's enums,
 * stencil_setup.h:26-43, riemann_solver_settings.h:47, enums/signal_speed.h:31,
 * enums/flux_splitting.h:31). Default: WENO5, Hllc, Einfeldt, Roe. Process-wide
 * setting: not to be changed while another thread runs a call. */
int oracle_set_options(int stencil, int riemann, int signal, int splitting);
/* TimeIntegrators (numerical_setup.h:26): RK2 = 0, RK3 = 1 (default). */
int oracle_set_time_integrator(int integrator);

/* cons = (mass, energy, mx, my, mz), prim = (rho, p, u, v, w);
 * out = pressure, enthalpy, energy, speed of sound, psi, gruneisen.
 * dim selects the dimension-aware sums as a DIMENSION=dim build does. */
int oracle_eos(int dim, double gamma, double B, int safe, const double *cons,
               const double *prim, double *out);

int oracle_prime_states(int dim, const double *u, int nb, double gamma,
                        double B, int safe, double *p);

int oracle_space_rhs(int dim, int solver, int recon, const double *u, int nb,
                     double gamma, double B, int safe, double cell_size,
                     double *fx, double *fy, double *fz, double *rhs,
                     int nthreads);

int oracle_timestep(int dim, const double *u, int nb, double gamma, double B,
                    int safe, double cell_size, double cfl, double t,
                    double t_end, double *dt);

int oracle_halo_fill(int dim, double *u, int nb, int nfields, const int *nbr26,
                     int faces_only, int zero_gradient);

/* six-face halo copy (W,E,S,N,B,T neighbour table, -1 = domain face) followed
 * by zero-gradient slabs on domain faces */
int oracle_halo_update(int dim, double *u, int nb, const int *nbr);

int oracle_run(int dim, int solver, int recon, double *u, int nb,
               const int *nbr, double gamma, double B, int safe,
               double cell_size, double cfl, double t_end, int max_steps,
               int nthreads, double *t_io, int *steps_done, double *dt_log);

/* Multi-level case: nleaf leaves, leaf b of level level[b] at integer node
 * coordinates coord[3b..3b+2] (units of its own node size) in a box of
 * n0[0] x n0[1] x n0[2] level-0 nodes with level-0 cell size h0; zero-gradient
 * domain faces. u [nleaf] blocks (interiors read and written). Local time
 * stepping over macro steps of 2^lmax micro steps; dt_log receives every
 * micro time step. Returns 0, or 4 (leaves do not tile the box) or 5 (face
 * neighbours more than one level apart). */
/* Multiresolution::Prediction (multiresolution.cpp:146-283) of one field
 * buffer [tc] into a child's cells start .. start + count (even numbers). */
int oracle_prediction(int dim, const double *parent, int octant, const int *start,
                      const int *count, double *child);
/* Face halos of every leaf of a multi-level snapshot (same-level copy, finer
 * neighbours averaged, coarser ones predicted), in place in u. */
int oracle_level_halos(int dim, double *u, int nleaf, const int *level, const int *coord,
                       const int *n0);
int oracle_levels_run(int dim, int solver, int recon, double *u, int nleaf,
                      const int *level, const int *coord, const int *n0, double h0,
                      double gamma, double B, int safe, double cfl, double t_end,
                      int max_macro, int nthreads, double *t_io, int *macro_done,
                      double *dt_log);

#ifdef __cplusplus
}
#endif
#endif
