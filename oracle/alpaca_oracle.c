/* TEST INFRASTRUCTURE ONLY — the CPU oracle, never part of the product path.
 *
 * Plain-C restatement of tumaer/ALPACA's per-block finite-volume right-hand
 * side, halo fill, CFL time step and SSP-RK3 stage update. Each function cites
 * the reference lines it restates (paths relative to ALPACA's src/). Every
 * multiply and add is written in the reference's association order, and the
 * file is compiled with -ffp-contract=off, so on the same inputs it reproduces
 * the reference compiled with the same flags bit for bit (checked by
 * tests/test_oracle.py against oracle/_ref, the reference's own sources built
 * by oracle/Makefile).
 *
 * Supported selections (user_specifications): EquationSet::Euler;
 * ConvectiveTermSolvers::FiniteVolume with StateReconstructionType::
 * Characteristic or Primitive, ReconstructionStencils::WENO5,
 * RiemannSolvers::Hllc and SignalSpeed::Einfeldt; ConvectiveTermSolvers::
 * FluxSplitting with FluxSplitting::Roe; TimeIntegrators::RK3; FUSY on;
 * StiffenedGas and StiffenedGasSafe.
 */
#include "alpaca_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define IC 16
#define HS 4
#define TC (IC + 2 * HS)
#define MAXNE 5

enum { MASS = 0, ENERGY = 1, MOMX = 2 };     /* field_setup.h:101-112 */
enum { RHO = 0, PRES = 1, VELX = 2 };        /* field_setup.h:114-130 */

typedef struct {
  int dim, ne, np;
  int tc[3], ic[3];
  long cells, faces;
} Geom;

static Geom make_geom(int dim) {
  Geom g;
  g.dim = dim;
  g.ne = dim + 2;
  g.np = dim + 2;
  for (int d = 0; d < 3; ++d) {
    g.tc[d] = d < dim ? TC : 1;
    g.ic[d] = d < dim ? IC : 1;
  }
  g.cells = (long)g.tc[0] * g.tc[1] * g.tc[2];
  g.faces = (long)(g.ic[0] + 1) * (g.ic[1] + 1) * (g.ic[2] + 1);
  return g;
}

static inline long cidx(const Geom *g, int i, int j, int k) {
  return ((long)i * g->tc[1] + j) * g->tc[2] + k;
}
static inline long fidx(const Geom *g, int i, int j, int k) {
  return ((long)i * (g->ic[1] + 1) + j) * (g->ic[2] + 1) + k;
}
/* first / last interior index per dimension (compile_time_constants.h:314-347) */
static inline int fic(const Geom *g, int d) { return d < g->dim ? HS : 0; }
static inline int lic(const Geom *g, int d) { return d < g->dim ? HS + IC - 1 : 0; }

typedef struct {
  int dim;
  double gamma, B;
  int safe;
} Eos;

/* std::min / std::max with the reference's tie behaviour */
static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static inline double dmax(double a, double b) { return (a < b) ? b : a; }

/* ConsistencyManagedSum with FUSY on (utilities/mathematical_functions.h:79-89) */
static double cms3(double a, double b, double c) {
  double const s1 = (a + b) + c;
  double const s2 = (a + c) + b;
  double const s3 = (b + c) + a;
  double mn = s1, mx = s1;
  if (s2 < mn) mn = s2;
  if (s3 < mn) mn = s3;
  if (mx < s2) mx = s2;
  if (mx < s3) mx = s3;
  return 0.5 * (mn + mx);
}

/* DimensionAwareConsistencyManagedSum (mathematical_functions.h:98-108) */
static inline double dacms(int dim, double a, double b, double c) {
  if (dim == 1) return a;
  if (dim == 2) return a + b;
  return cms3(a, b, c);
}

/* ConsistencyManagedSum(std::array<double, DIM>) (mathematical_functions.h:130-150) */
static inline double cms_array(int dim, const double *v) {
  if (dim == 1) return v[0];
  if (dim == 2) return v[0] + v[1];
  return cms3(v[0], v[1], v[2]);
}

/* ---- equation of state ------------------------------------------------- */

/* GenericStiffenedGas::CalculatePressure<false> (generic_stiffened_gas.h:40-57),
 * StiffenedGasSafe::ComputePressure (stiffened_gas_safe.cpp:61-75) */
static double eos_pressure(const Eos *e, double mass, double mx, double my,
                           double mz, double energy) {
  if (e->safe) {
    double const p = -e->gamma * e->B +
                     (e->gamma - 1.0) *
                         (energy - 0.5 * dacms(e->dim, mx * mx, my * my, mz * mz) /
                                       dmax(mass, DBL_EPSILON));
    return dmax(p, -e->B + DBL_EPSILON);
  }
  double const q = 0.5 * dacms(e->dim, mx * mx, my * my, mz * mz);
  return -e->gamma * e->B + (e->gamma - 1.0) * (energy - q / mass);
}

/* StiffenedGas::ComputeEnthalpy (stiffened_gas.cpp:88-96), safe: stiffened_gas_safe.cpp:77-84 */
static double eos_enthalpy(const Eos *e, double mass, double mx, double my,
                           double mz, double energy) {
  double const p = eos_pressure(e, mass, mx, my, mz, energy);
  if (e->safe) return (energy + p) / dmax(mass, DBL_EPSILON);
  return (energy + p) / mass;
}

/* GenericStiffenedGas::CalculateEnergy (generic_stiffened_gas.h:70-79) */
static double eos_energy(const Eos *e, double rho, double u, double v, double w,
                         double p) {
  return (p + e->gamma * e->B) / (e->gamma - 1.0) +
         (0.5 * dacms(e->dim, u * u, v * v, w * w) * rho);
}

/* GenericStiffenedGas::CalculateSpeedOfSound (generic_stiffened_gas.h:90-102),
 * StiffenedGasSafe::ComputeSpeedOfSound (stiffened_gas_safe.cpp:140-146) */
static double eos_speed_of_sound(const Eos *e, double rho, double p) {
  if (e->safe) {
    double const c2 = e->gamma * (p + e->B) / dmax(rho, DBL_EPSILON);
    return sqrt(dmax(c2, DBL_EPSILON));
  }
  return sqrt(e->gamma * (p + e->B) / rho);
}

/* StiffenedGas::ComputePsi (stiffened_gas.cpp:133-136) */
static inline double eos_psi(const Eos *e, double p, double one_rho) {
  return (p + e->gamma * e->B) * one_rho;
}

/* StiffenedGas::GetGruneisen (stiffened_gas.cpp:113) */
static inline double eos_gruneisen(const Eos *e) { return e->gamma - 1.0; }

/* ConservativesToPrimeStates (prime_state_handler.h:277-371), Euler set */
static void cons_to_prim(const Eos *e, const double *c, double *p) {
  int const dim = e->dim;
  p[RHO] = c[MASS];
  double const one_density = 1.0 / c[MASS];
  for (int d = 0; d < dim; ++d) p[VELX + d] = c[MOMX + d] * one_density;
  p[PRES] = eos_pressure(e, c[MASS], c[MOMX], dim > 1 ? c[MOMX + 1] : 0.0,
                         dim > 2 ? c[MOMX + 2] : 0.0, c[ENERGY]);
}

/* PrimeStatesToConservatives (prime_state_handler.h:195-275), Euler set */
static void prim_to_cons(const Eos *e, const double *p, double *c) {
  int const dim = e->dim;
  c[MASS] = p[RHO];
  for (int d = 0; d < dim; ++d) c[MOMX + d] = p[VELX + d] * p[RHO];
  c[ENERGY] = eos_energy(e, p[RHO], p[VELX], dim > 1 ? p[VELX + 1] : 0.0,
                         dim > 2 ? p[VELX + 2] : 0.0, p[PRES]);
}

/* ---- WENO5-JS (stencils/spatial_reconstruction_stencils/weno5.h:88-158) -- */

/* evaluation properties {offset, sign}: UpwindLeft {0,1}, UpwindRight {1,-1}
 * (stencils/apply_wrapper.h:47-57); downstream stencil size 2. */
static double weno5(const double *a, int offset, int sign) {
  double const v1 = a[2 + offset - 2 * sign];
  double const v2 = a[2 + offset - 1 * sign];
  double const v3 = a[2 + offset];
  double const v4 = a[2 + offset + 1 * sign];
  double const v5 = a[2 + offset + 2 * sign];
  double const c1 = 13.0 / 12.0, c2 = 0.25;

  double const s11 = 1.0 * v1 + -2.0 * v2 + 1.0 * v3;
  double const s12 = 1.0 * v1 + -4.0 * v2 + 3.0 * v3;
  double const s1 = c1 * s11 * s11 + c2 * s12 * s12;
  double const s21 = 1.0 * v2 + -2.0 * v3 + 1.0 * v4;
  double const s22 = 1.0 * v2 + -1.0 * v4;
  double const s2 = c1 * s21 * s21 + c2 * s22 * s22;
  double const s31 = 1.0 * v3 + -2.0 * v4 + 1.0 * v5;
  double const s32 = 3.0 * v3 + -4.0 * v4 + 1.0 * v5;
  double const s3 = c1 * s31 * s31 + c2 * s32 * s32;

  double const eps = 1.0e-6;
  double const a1 = 0.1 / ((s1 + eps) * (s1 + eps));
  double const a2 = 0.6 / ((s2 + eps) * (s2 + eps));
  double const a3 = 0.3 / ((s3 + eps) * (s3 + eps));
  double const one_a_sum = 1.0 / (a1 + a2 + a3);
  double const w1 = a1 * one_a_sum;
  double const w2 = a2 * one_a_sum;
  double const w3 = a3 * one_a_sum;

  return w1 * (2.0 / 6.0 * v1 + -7.0 / 6.0 * v2 + 11.0 / 6.0 * v3) +
         w2 * (-1.0 / 6.0 * v2 + 5.0 / 6.0 * v3 + 2.0 / 6.0 * v4) +
         w3 * (2.0 / 6.0 * v3 + 5.0 / 6.0 * v4 + -1.0 / 6.0 * v5);
}
static inline double weno5_left(const double *a) { return weno5(a, 0, 1); }
static inline double weno5_right(const double *a) { return weno5(a, 1, -1); }

/* ---- further selections of the plugin surface (enum values of the
 * reference: stencil_setup.h:26-43, riemann_solver_settings.h:47,
 * enums/signal_speed.h:31, enums/flux_splitting.h:31) -------------------- */
enum { ST_FIRST_ORDER = 0, ST_WENO3 = 1, ST_WENO5 = 4, ST_WENO5Z = 7, ST_TENO5 = 11,
       ST_WENO7 = 13 };
#define MAXW 8 /* widest stencil: WENO7, cells i-3 .. i+4 */
enum { RS_HLLC = 0, RS_HLLC_LM = 1, RS_HLL = 2 };
enum { SS_EINFELDT = 0, SS_DAVIS = 1, SS_TORO = 2, SS_ARITHMETIC = 3 };
enum { FSP_ROE = 0, FSP_LLF = 1, FSP_GLF = 2, FSP_ROE_M = 3, FSP_LLF_M = 4 };
static int g_stencil = ST_WENO5, g_riemann = RS_HLLC, g_signal = SS_EINFELDT,
           g_splitting = FSP_ROE;
static double g_glf[3]; /* global Lax-Friedrichs wave speeds (glf_maxima) */

/* WENO5-Z (weno5_z.h:88-150) */
static double weno5z(const double *a, int offset, int sign) {
  double const v1 = a[2 + offset - 2 * sign];
  double const v2 = a[2 + offset - 1 * sign];
  double const v3 = a[2 + offset];
  double const v4 = a[2 + offset + 1 * sign];
  double const v5 = a[2 + offset + 2 * sign];
  double const c1 = 13.0 / 12.0, c2 = 0.25;
  double const s11 = 1.0 * v1 + -2.0 * v2 + 1.0 * v3;
  double const s12 = 1.0 * v1 + -4.0 * v2 + 3.0 * v3;
  double const s1 = c1 * s11 * s11 + c2 * s12 * s12;
  double const s21 = 1.0 * v2 + -2.0 * v3 + 1.0 * v4;
  double const s22 = 1.0 * v2 + -1.0 * v4;
  double const s2 = c1 * s21 * s21 + c2 * s22 * s22;
  double const s31 = 1.0 * v3 + -2.0 * v4 + 1.0 * v5;
  double const s32 = 3.0 * v3 + -4.0 * v4 + 1.0 * v5;
  double const s3 = c1 * s31 * s31 + c2 * s32 * s32;
  double const tau = fabs(s1 - s3);
  double const a1 = 0.1 * (1.0 + tau / (s1 + DBL_EPSILON));
  double const a2 = 0.6 * (1.0 + tau / (s2 + DBL_EPSILON));
  double const a3 = 0.3 * (1.0 + tau / (s3 + DBL_EPSILON));
  double const one_a_sum = 1.0 / (a1 + a2 + a3);
  double const w1 = a1 * one_a_sum, w2 = a2 * one_a_sum, w3 = a3 * one_a_sum;
  return w1 * (2.0 / 6.0 * v1 + -7.0 / 6.0 * v2 + 11.0 / 6.0 * v3) +
         w2 * (-1.0 / 6.0 * v2 + 5.0 / 6.0 * v3 + 2.0 / 6.0 * v4) +
         w3 * (2.0 / 6.0 * v3 + 5.0 / 6.0 * v4 + -1.0 / 6.0 * v5);
}

/* TENO5 (teno5.h:98-180), cut-off C_T = 1e-5 */
static double teno5(const double *a, int offset, int sign) {
  double const v1 = a[2 + offset - 2 * sign];
  double const v2 = a[2 + offset - 1 * sign];
  double const v3 = a[2 + offset];
  double const v4 = a[2 + offset + 1 * sign];
  double const v5 = a[2 + offset + 2 * sign];
  double const c1 = 13.0 / 12.0, c2 = 0.25;
  double const s11 = 1.0 * v2 + -2.0 * v3 + 1.0 * v4;
  double const s12 = 1.0 * v2 + -1.0 * v4;
  double const s1 = c1 * s11 * s11 + c2 * s12 * s12;
  double const s21 = 1.0 * v3 + -2.0 * v4 + 1.0 * v5;
  double const s22 = 3.0 * v3 + -4.0 * v4 + 1.0 * v5;
  double const s2 = c1 * s21 * s21 + c2 * s22 * s22;
  double const s31 = 1.0 * v1 + -2.0 * v2 + 1.0 * v3;
  double const s32 = 1.0 * v1 + -4.0 * v2 + 3.0 * v3;
  double const s3 = c1 * s31 * s31 + c2 * s32 * s32;
  double const tau5 = fabs(s3 - s2);
  double a1 = 1.0 + tau5 / (s1 + DBL_EPSILON);
  double a2 = 1.0 + tau5 / (s2 + DBL_EPSILON);
  double a3 = 1.0 + tau5 / (s3 + DBL_EPSILON);
  a1 *= (a1 * a1);
  a2 *= (a2 * a2);
  a3 *= (a3 * a3);
  a1 *= a1;
  a2 *= a2;
  a3 *= a3;
  double const one_a_sum = 1.0 / (a1 + a2 + a3);
  double const b1 = a1 * one_a_sum < 1.0e-5 ? 0.0 : 1.0;
  double const b2 = a2 * one_a_sum < 1.0e-5 ? 0.0 : 1.0;
  double const b3 = a3 * one_a_sum < 1.0e-5 ? 0.0 : 1.0;
  double const var1 = -1.0 * v2 + 5.0 * v3 + 2.0 * v4;
  double const var2 = 2.0 * v3 + 5.0 * v4 + -1.0 * v5;
  double const var3 = 2.0 * v1 + -7.0 * v2 + 11.0 * v3;
  double const w1 = 0.6 * b1, w2 = 0.3 * b2, w3 = 0.1 * b3;
  double const one_w_sum = 1.0 / (w1 + w2 + w3);
  return (w1 * one_w_sum * var1 + w2 * one_w_sum * var2 + w3 * one_w_sum * var3) * (1.0 / 6.0);
}

/* WENO3 (weno3.h:66-100): cells i-1..i+2 are a[1..4]; downstream size 1 */
static double weno3(const double *a, int offset, int sign) {
  double const v1 = a[2 + offset - 1 * sign];
  double const v2 = a[2 + offset];
  double const v3 = a[2 + offset + 1 * sign];
  double const s11 = -1.0 * v1 + 1.0 * v2;
  double const s1 = s11 * s11;
  double const s21 = -1.0 * v2 + 1.0 * v3;
  double const s2 = s21 * s21;
  double const a1 = (1.0 / 3.0) / ((s1 + DBL_EPSILON) * (s1 + DBL_EPSILON));
  double const a2 = (2.0 / 3.0) / ((s2 + DBL_EPSILON) * (s2 + DBL_EPSILON));
  double const one_a_sum = 1.0 / (a1 + a2);
  double const w1 = a1 * one_a_sum, w2 = a2 * one_a_sum;
  return w1 * (-1.0 / 2.0 * v1 + 3.0 / 2.0 * v2) + w2 * (1.0 / 2.0 * v2 + 1.0 / 2.0 * v3);
}

/* WENO7-JS (stencils/spatial_reconstruction_stencils/weno7.h:21-212; the
 * coefficients of Balsara & Shu 2000): a[0..7] are cells i-3..i+4 around face
 * i+1/2 (downstream stencil size 3), eps 1e-10. */
static double weno7(const double *a, int offset, int sign) {
  double const v1 = a[3 + offset - 3 * sign];
  double const v2 = a[3 + offset - 2 * sign];
  double const v3 = a[3 + offset - 1 * sign];
  double const v4 = a[3 + offset];
  double const v5 = a[3 + offset + 1 * sign];
  double const v6 = a[3 + offset + 2 * sign];
  double const v7 = a[3 + offset + 3 * sign];
  double const s11 = 547.0 * v1 + -3882.0 * v2 + 4642.0 * v3 + -1854.0 * v4;
  double const s12 = 7043.0 * v2 + -17246.0 * v3 + 7042.0 * v4;
  double const s13 = 11003.0 * v3 + -9402.0 * v4;
  double const s14 = 2107.0 * v4;
  double const s1 = v1 * s11 + v2 * s12 + v3 * s13 + v4 * s14;
  double const s21 = 267.0 * v2 + -1642.0 * v3 + 1602.0 * v4 + -494.0 * v5;
  double const s22 = 2843.0 * v3 + -5966.0 * v4 + 1922.0 * v5;
  double const s23 = 3443.0 * v4 + -2522.0 * v5;
  double const s24 = 547.0 * v5;
  double const s2 = v2 * s21 + v3 * s22 + v4 * s23 + v5 * s24;
  double const s31 = 547.0 * v3 + -2522.0 * v4 + 1922.0 * v5 + -494.0 * v6;
  double const s32 = 3443.0 * v4 + -5966.0 * v5 + 1602.0 * v6;
  double const s33 = 2843.0 * v5 + -1642.0 * v6;
  double const s34 = 267.0 * v6;
  double const s3 = v3 * s31 + v4 * s32 + v5 * s33 + v6 * s34;
  double const s41 = 2107.0 * v4 + -9402.0 * v5 + 7042.0 * v6 + -1854.0 * v7;
  double const s42 = 11003.0 * v5 + -17246.0 * v6 + 4642.0 * v7;
  double const s43 = 7043.0 * v6 + -3882.0 * v7;
  double const s44 = 547.0 * v7;
  double const s4 = v4 * s41 + v5 * s42 + v6 * s43 + v7 * s44;
  double const eps = 1.0e-10;
  double const a1 = (1.0 / 35.0) / ((s1 + eps) * (s1 + eps));
  double const a2 = (12.0 / 35.0) / ((s2 + eps) * (s2 + eps));
  double const a3 = (18.0 / 35.0) / ((s3 + eps) * (s3 + eps));
  double const a4 = (4.0 / 35.0) / ((s4 + eps) * (s4 + eps));
  double const one_a_sum = 1.0 / (a1 + a2 + a3 + a4);
  double const w1 = a1 * one_a_sum, w2 = a2 * one_a_sum, w3 = a3 * one_a_sum,
               w4 = a4 * one_a_sum;
  return w1 * (-3.0 / 12.0 * v1 + 13.0 / 12.0 * v2 + -23.0 / 12.0 * v3 + 25.0 / 12.0 * v4) +
         w2 * (1.0 / 12.0 * v2 + -5.0 / 12.0 * v3 + 13.0 / 12.0 * v4 + 3.0 / 12.0 * v5) +
         w3 * (-1.0 / 12.0 * v3 + 7.0 / 12.0 * v4 + 7.0 / 12.0 * v5 + -1.0 / 12.0 * v6) +
         w4 * (3.0 / 12.0 * v4 + 13.0 / 12.0 * v5 + -5.0 / 12.0 * v6 + 1.0 / 12.0 * v7);
}

/* Cells of the selected stencil around face i+1/2 (the reference's
 * stencil_size_): 8 for WENO7 (cell i at index 3), else 6 (cell i at 2). */
static int stencil_width(void) { return g_stencil == ST_WENO7 ? 8 : 6; }

/* SU::Reconstruction with the selected stencil (stencils/stencil_utilities.h),
 * UpwindLeft {0, 1} / UpwindRight {1, -1}; FirstOrder returns cell i / i+1.
 * a holds stencil_width() cells. */
static double recon(const double *a, int offset, int sign) {
  switch (g_stencil) {
    case ST_WENO7: return weno7(a, offset, sign);
    case ST_WENO5Z: return weno5z(a, offset, sign);
    case ST_TENO5: return teno5(a, offset, sign);
    case ST_WENO3: return weno3(a, offset, sign);
    case ST_FIRST_ORDER: return a[2 + offset];
    default: return weno5(a, offset, sign);
  }
}
static inline double recon_left(const double *a) { return recon(a, 0, 1); }
static inline double recon_right(const double *a) { return recon(a, 1, -1); }

/* ---- Roe eigensystem (solvers/eigendecomposition.h:181-467) ------------ */

/* minor directions (eigendecomposition.h:84-125) */
static inline int minor_dir(int dir, int m) {
  static const int tab[3][2] = {{1, 2}, {0, 2}, {0, 1}};
  return tab[dir][m];
}

/* symmetry-preserving summation sequences
 * (solvers/state_reconstruction/state_reconstruction.h:35-58) */
static const int *summation_sequence(int dim, int dir) {
  static const int s1[3] = {MOMX, MASS, ENERGY};
  static const int s2[4] = {MOMX, MOMX + 1, MASS, ENERGY};
  static const int s3[3][5] = {{MOMX + 1, MOMX + 2, MOMX, MASS, ENERGY},
                               {MOMX + 2, MOMX, MOMX + 1, MASS, ENERGY},
                               {MOMX, MOMX + 1, MOMX + 2, MASS, ENERGY}};
  if (dim == 1) return s1;
  if (dim == 2) return s2;
  return s3[dir];
}

typedef struct {
  double L[MAXNE][MAXNE];
  double R[MAXNE][MAXNE];
  double ev[MAXNE];
} Eigen;

/* One face of ComputeRoeEigendecomposition<DIR> between cell t and neighbour n.
 * u: conservatives of the block, p: prime states of the block. Leaves the
 * output untouched when a density is non-positive (eigendecomposition.h:244). */
static void roe_eigen(const Geom *g, const Eos *e, int dir, const double *u,
                      const double *p, long t, long n, Eigen *out) {
  int const dim = g->dim, ne = g->ne;
  long const C = g->cells;
  double const rho_t = u[MASS * C + t], rho_n = u[MASS * C + n];
  if (rho_t <= 0.0 || rho_n <= 0.0) return;
  int const principal = dir;
  int const minor1 = dim > 1 ? minor_dir(dir, 0) : 0;
  int const minor2 = dim > 2 ? minor_dir(dir, 1) : 0;
  int const ev_principal = dim;
  double const gru = eos_gruneisen(e);

  double const one_rho_t = 1.0 / rho_t;
  double const energy_t = u[ENERGY * C + t];
  double const mx_t = u[MOMX * C + t];
  double const my_t = dim > 1 ? u[(MOMX + 1) * C + t] : 0.0;
  double const mz_t = dim > 2 ? u[(MOMX + 2) * C + t] : 0.0;
  double const up_t = p[(VELX + principal) * C + t];
  double const u1_t = dim > 1 ? p[(VELX + minor1) * C + t] : 0.0;
  double const u2_t = dim > 2 ? p[(VELX + minor2) * C + t] : 0.0;
  double const p_t = p[PRES * C + t];
  double const psi_t = eos_psi(e, p_t, one_rho_t);

  double const one_rho_n = 1.0 / rho_n;
  double const energy_n = u[ENERGY * C + n];
  double const mx_n = u[MOMX * C + n];
  double const my_n = dim > 1 ? u[(MOMX + 1) * C + n] : 0.0;
  double const mz_n = dim > 2 ? u[(MOMX + 2) * C + n] : 0.0;
  double const up_n = p[(VELX + principal) * C + n];
  double const u1_n = dim > 1 ? p[(VELX + minor1) * C + n] : 0.0;
  double const u2_n = dim > 2 ? p[(VELX + minor2) * C + n] : 0.0;
  double const p_n = p[PRES * C + n];
  double const psi_n = eos_psi(e, p_n, one_rho_n);

  double const sr_t = sqrt(rho_t);
  double const sr_n = sqrt(rho_n);
  double const rho_div = 1.0 / (sr_t + sr_n);
  double const rho_roe = sr_t * sr_n;
  double const one_rho_roe = 1.0 / rho_roe;

  double const up = ((up_t * sr_t) + (up_n * sr_n)) * rho_div;
  double const u1 = ((u1_t * sr_t) + (u1_n * sr_n)) * rho_div;
  double const u2 = ((u2_t * sr_t) + (u2_n * sr_n)) * rho_div;
  double const psi = ((psi_t * sr_t) + (psi_n * sr_n)) * rho_div;
  double const H = (eos_enthalpy(e, rho_t, mx_t, my_t, mz_t, energy_t) * sr_t +
                    eos_enthalpy(e, rho_n, mx_n, my_n, mz_n, energy_n) * sr_n) *
                   rho_div;

  double const q2 = dacms(dim, up * up, u1 * u1, u2 * u2);
  double const tmp = dacms(dim, (up_t - up_n) * (up_t - up_n),
                           (u1_t - u1_n) * (u1_t - u1_n),
                           (u2_t - u2_n) * (u2_t - u2_n));
  double const p_over_rho =
      ((p_t * one_rho_t) * sr_t + (p_n * one_rho_n) * sr_n) * rho_div +
      0.5 * rho_roe * (rho_div * rho_div) * tmp;
  double const cc = psi + gru * p_over_rho;
  double const one_cc = 1.0 / cc;
  double const c = sqrt(cc);

  int const mP = MOMX + principal, m1 = MOMX + minor1, m2 = MOMX + minor2;
  double(*L)[MAXNE] = out->L;
  double(*R)[MAXNE] = out->R;

  /* left eigenvectors (eigendecomposition.h:316-359) */
  L[0][MASS] = 0.5 * one_cc * (gru * q2 - gru * H + (up + c) * c);
  L[0][mP] = 0.5 * one_cc * (-up * gru - c);
  if (dim > 1) L[0][m1] = 0.5 * one_cc * (-u1 * gru);
  if (dim > 2) L[0][m2] = 0.5 * one_cc * (-u2 * gru);
  L[0][ENERGY] = 0.5 * one_cc * gru;
  if (dim > 1) {
    L[1][MASS] = u1 * one_rho_roe;
    L[1][mP] = 0.0;
    L[1][m1] = -one_rho_roe;
    if (dim > 2) L[1][m2] = 0.0;
    L[1][ENERGY] = 0.0;
  }
  if (dim > 2) {
    L[2][MASS] = -u2 * one_rho_roe;
    L[2][mP] = 0.0;
    L[2][m1] = 0.0;
    L[2][m2] = one_rho_roe;
    L[2][ENERGY] = 0.0;
  }
  L[ev_principal][MASS] = one_cc * (H - q2);
  L[ev_principal][mP] = one_cc * up;
  if (dim > 1) L[ev_principal][m1] = one_cc * u1;
  if (dim > 2) L[ev_principal][m2] = one_cc * u2;
  L[ev_principal][ENERGY] = -one_cc;
  L[ne - 1][MASS] = 0.5 * one_cc * (gru * q2 - gru * H - (up - c) * c);
  L[ne - 1][mP] = 0.5 * one_cc * (-up * gru + c);
  if (dim > 1) L[ne - 1][m1] = 0.5 * one_cc * (-u1 * gru);
  if (dim > 2) L[ne - 1][m2] = 0.5 * one_cc * (-u2 * gru);
  L[ne - 1][ENERGY] = 0.5 * one_cc * gru;

  /* right eigenvectors (eigendecomposition.h:366-409) */
  R[MASS][0] = 1.0;
  if (dim > 1) R[MASS][1] = 0.0;
  if (dim > 2) R[MASS][2] = 0.0;
  R[MASS][ev_principal] = gru;
  R[MASS][ne - 1] = 1.0;
  R[mP][0] = up - c;
  if (dim > 1) R[mP][1] = 0.0;
  if (dim > 2) R[mP][2] = 0.0;
  R[mP][ev_principal] = gru * up;
  R[mP][ne - 1] = up + c;
  if (dim > 1) {
    R[m1][0] = u1;
    R[m1][1] = -rho_roe;
    if (dim > 2) R[m1][2] = 0.0;
    R[m1][ev_principal] = gru * u1;
    R[m1][ne - 1] = u1;
  }
  if (dim > 2) {
    R[m2][0] = u2;
    R[m2][1] = 0.0;
    R[m2][2] = rho_roe;
    R[m2][ev_principal] = gru * u2;
    R[m2][ne - 1] = u2;
  }
  R[ENERGY][0] = H - up * c;
  if (dim > 1) R[ENERGY][1] = -u1 * rho_roe;
  if (dim > 2) R[ENERGY][2] = rho_roe * u2;
  R[ENERGY][ev_principal] = gru * H - c * c;
  R[ENERGY][ne - 1] = H + up * c;

  /* flux-splitting wave speeds (eigendecomposition.h:416-454, 64-72): Roe,
   * Roe-M, local Lax-Friedrichs, LLF-M; low-Mach limit factor 5 */
  double e0, elin, e1;
  if (g_splitting == FSP_ROE_M) {
    double const cm = dmin(c, 5.0 * fabs(up));
    e0 = fabs(up - cm);
    elin = fabs(up);
    e1 = fabs(up + cm);
  } else if (g_splitting == FSP_GLF) {
    /* the x maxima in every direction (eigendecomposition.h:457-460) */
    e0 = g_glf[0];
    elin = g_glf[1];
    e1 = g_glf[2];
  } else if (g_splitting == FSP_LLF || g_splitting == FSP_LLF_M) {
    double ct = eos_speed_of_sound(e, rho_t, p_t);
    double cn = eos_speed_of_sound(e, rho_n, p_n);
    if (g_splitting == FSP_LLF_M) {
      ct = dmin(5.0 * fabs(up_t), ct);
      cn = dmin(5.0 * fabs(up_n), cn);
    }
    e0 = dmax(fabs(up_t - ct), fabs(up_n - cn));
    elin = dmax(fabs(up_t), fabs(up_n));
    e1 = dmax(fabs(up_t + ct), fabs(up_n + cn));
  } else {
    e0 = fabs(up - c);
    elin = fabs(up);
    e1 = fabs(up + c);
  }
  out->ev[0] = e0;
  out->ev[ne - 1] = e1;
  for (int l = 1; l < ne - 1; ++l) out->ev[l] = elin;
}

/* TransformToPhysicalSpace (eigendecomposition.h:144-165) */
static void to_physical(int ne, const double *ch, double R[MAXNE][MAXNE],
                        double *out) {
  for (int l = 0; l < ne; ++l) {
    out[l] = 0.0;
    for (int n = 1; n < ne - 1; ++n) out[l] += ch[n] * R[l][n];
    out[l] += (ch[0] * R[l][0] + ch[ne - 1] * R[l][ne - 1]);
  }
}

/* ---- HLL-type Riemann solvers and their signal speeds ------------------ */

/* CalculateSignalSpeed, Einfeldt branch (hll_signal_speed_calculator.h:77-101) */
static void einfeldt(double rl, double rr, double ul, double ur, double cl,
                     double cr, double *sl, double *sr) {
  double const srl = sqrt(rl);
  double const srr = sqrt(rr);
  double const rho_div = 1.0 / (srl + srr);
  double const u_roe = ((ul * srl) + (ur * srr)) * rho_div;
  double const c_e = sqrt(((cl * cl * srl) + (cr * cr * srr)) * rho_div +
                          (0.5 * srl * srr * rho_div * rho_div) * (ur - ul) *
                              (ur - ul));
  *sl = dmin(u_roe - c_e, ul - cl);
  *sr = dmax(u_roe + c_e, ur + cr);
}

/* CalculateSignalSpeed, the other branches (hll_signal_speed_calculator.h:40-140) */
static void signal_speeds(double rl, double rr, double ul, double ur, double pl,
                          double pr, double cl, double cr, double gamma, double *sl,
                          double *sr) {
  if (g_signal == SS_ARITHMETIC) {
    double const cf = 0.5 * (cl + cr);
    double const uf = 0.5 * (ul + ur);
    *sl = dmin(uf - cf, ul - cl);
    *sr = dmax(uf + cf, ur + cr);
  } else if (g_signal == SS_DAVIS) {
    *sl = dmin(ul - cl, ur - cr);
    *sr = dmax(ul + cl, ur + cr);
  } else if (g_signal == SS_TORO) {
    double const z = (gamma - 1.0) / (2.0 * gamma);
    double const p_star =
        pow(((cl + cr) - 0.5 * (ur - ul) * (gamma - 1.0)) / (cl / pow(pl, z) + cr / pow(pr, z)),
            (1.0 / z));
    double ql = 1.0, qr = 1.0;
    if (p_star > pl) ql = sqrt(1.0 + (gamma + 1.0) / (2.0 * gamma) * (p_star / pl - 1.0));
    if (p_star > pr) qr = sqrt(1.0 + (gamma + 1.0) / (2.0 * gamma) * (p_star / pr - 1.0));
    *sl = ul - cl * ql;
    *sr = ur + cr * qr;
  } else {
    einfeldt(rl, rr, ul, ur, cl, cr, sl, sr);
  }
}

static inline int signum(double x) { return (0.0 < x) - (x < 0.0); }

/* HllcRiemannSolver::SolveRiemannProblemImplementation
 * (riemann_solvers/hllc_riemann_solver.h:52-198), or with the selection
 * g_riemann the HLL or HLLC-LM solver; signal speeds per g_signal. */
static void hllc(const Eos *e, int dir, const double *cl, const double *cr,
                 const double *pl, const double *pr, double *flux) {
  int const dim = e->dim, ne = dim + 2;
  int const mP = MOMX + dir, vP = VELX + dir;
  double qsl[MAXNE], qsr[MAXNE], fl[MAXNE], fr[MAXNE];

  double const pres_l = pl[PRES], pres_r = pr[PRES];
  double const one_rl = 1.0 / cl[MASS], one_rr = 1.0 / cr[MASS];
  double const vel_l = pl[vP], vel_r = pr[vP];
  double const c_l = eos_speed_of_sound(e, cl[MASS], pres_l);
  double const c_r = eos_speed_of_sound(e, cr[MASS], pres_r);
  double sls, srs;
  signal_speeds(cl[MASS], cr[MASS], vel_l, vel_r, pres_l, pres_r, c_l, c_r, e->gamma, &sls, &srs);
  fl[MASS] = cl[mP];
  fl[mP] = ((cl[mP] * cl[mP]) * one_rl) + pres_l;
  fl[ENERGY] = vel_l * (cl[ENERGY] + pres_l);
  fr[MASS] = cr[mP];
  fr[mP] = ((cr[mP] * cr[mP]) * one_rr) + pres_r;
  fr[ENERGY] = vel_r * (cr[ENERGY] + pres_r);
  for (int d = 0; d < dim - 1; ++d) {
    int const mm = MOMX + minor_dir(dir, d);
    fl[mm] = vel_l * cl[mm];
    fr[mm] = vel_r * cr[mm];
  }
  if (g_riemann == RS_HLL) {
    /* HllRiemannSolver (hll_riemann_solver.h:96-150) */
    double const sl = dmin(sls, 0.0), sr = dmax(srs, 0.0);
    for (int n = 0; n < ne; ++n)
      flux[n] = (((sr * fl[n]) - (sl * fr[n])) + ((sr * sl) * (cr[n] - cl[n]))) / (sr - sl);
    return;
  }
  int const lm = g_riemann == RS_HLLC_LM; /* HllcLMRiemannSolver: unclamped speeds */
  double const s_star =
      ((pres_r - pres_l) + (cl[mP] * (sls - vel_l) - cr[mP] * (srs - vel_r))) /
      (cl[MASS] * (sls - vel_l) - cr[MASS] * (srs - vel_r));
  double const sl = lm ? sls : dmin(sls, 0.0);
  double const sr = lm ? srs : dmax(srs, 0.0);
  double const chi_l = (sls - vel_l) / (sls - s_star);
  double const chi_r = (srs - vel_r) / (srs - s_star);

  qsl[MASS] = cl[MASS] * chi_l;
  qsl[mP] = cl[MASS] * chi_l * s_star;
  qsl[ENERGY] = cl[MASS] * chi_l *
                (cl[ENERGY] * one_rl +
                 (s_star - vel_l) * (s_star + pres_l / (cl[MASS] * (sl - vel_l))));
  qsr[MASS] = cr[MASS] * chi_r;
  qsr[mP] = cr[MASS] * chi_r * s_star;
  qsr[ENERGY] = cr[MASS] * chi_r *
                (cr[ENERGY] * one_rr +
                 (s_star - vel_r) * (s_star + pres_r / (cr[MASS] * (sr - vel_r))));

  for (int d = 0; d < dim - 1; ++d) {
    int const mm = MOMX + minor_dir(dir, d);
    qsl[mm] = chi_l * cl[mm];
    qsr[mm] = chi_r * cr[mm];
  }
  if (lm) {
    /* low-Mach activation (hllc_lm_riemann_solver.h:180-198), Ma limit 0.1 */
    double const ma = dmin(0.1, dmax(fabs(vel_l / c_l), fabs(vel_r / c_r)));
    double const act = sin((ma / 0.1) * 1.57079632679489661923);
    for (int n = 0; n < ne; ++n) {
      if (sl >= 0.0)
        flux[n] = fl[n];
      else if (sr <= 0.0)
        flux[n] = fr[n];
      else
        flux[n] = 0.5 * ((fl[n] + fr[n]) - (((act * sr) * (cr[n] - qsr[n]) +
                                             (act * sl) * (cl[n] - qsl[n])) +
                                            fabs(s_star) * (qsr[n] - qsl[n])));
    }
    return;
  }
  int const sg = signum(s_star);
  for (int n = 0; n < ne; ++n) {
    double const fsl = fl[n] + (sl * (qsl[n] - cl[n]));
    double const fsr = fr[n] + (sr * (qsr[n] - cr[n]));
    flux[n] = (0.5 * (1.0 + sg) * fsl + 0.5 * (1.0 - sg) * fsr);
  }
}

/* ---- per-block right-hand side ----------------------------------------- */

typedef struct {
  double *prim;   /* [np][cells] */
  Eigen *eig;     /* [faces] */
  double *adv;    /* [ne][cells] (flux splitting) */
} Work;

static void work_alloc(const Geom *g, Work *w) {
  w->prim = (double *)malloc(sizeof(double) * g->np * g->cells);
  w->eig = (Eigen *)malloc(sizeof(Eigen) * g->faces);
  w->adv = (double *)malloc(sizeof(double) * g->ne * g->cells);
}
static void work_free(Work *w) {
  free(w->prim);
  free(w->eig);
  free(w->adv);
}

/* block-wide prime states (prime_state_handler.h:141-152) */
/* Global Lax-Friedrichs wave speeds: the largest |u - c|, |u|, |u + c| of the
 * x velocity over the interior cells of all blocks whose density is positive
 * (EigenDecomposition::ComputeMaxEigenvaluesOnBlock, eigendecomposition.cpp:
 * 46-110; maxima across blocks before the fluxes of every stage in
 * ComputeRightHandSide, modular_algorithm_assembler.cpp:957-985). Only the x
 * maxima are kept (g_glf): the flux uses them in every direction. */

static void glf_maxima(const Geom *g, const Eos *e, const double *u, int nb) {
  double m[3] = {0.0, 0.0, 0.0};
  double c[MAXNE], p[MAXNE];
  for (int b = 0; b < nb; ++b) {
    const double *ub = u + (long)b * g->ne * g->cells;
    for (int i = fic(g, 0); i <= lic(g, 0); ++i)
      for (int j = fic(g, 1); j <= lic(g, 1); ++j)
        for (int k = fic(g, 2); k <= lic(g, 2); ++k) {
          long const x = cidx(g, i, j, k);
          for (int f = 0; f < g->ne; ++f) c[f] = ub[f * g->cells + x];
          cons_to_prim(e, c, p);
          if (p[RHO] <= 0.0) continue;
          double const cs = eos_speed_of_sound(e, p[RHO], p[PRES]);
          double const vx = p[VELX];
          m[0] = dmax(m[0], fabs(vx - cs));
          m[1] = dmax(m[1], fabs(vx));
          m[2] = dmax(m[2], fabs(vx + cs));
        }
  }
  for (int q = 0; q < 3; ++q) g_glf[q] = m[q];
}

/* The same maxima over the leaves items[0..ni) whose right-hand side is
 * computed (ComputeRightHandSide takes them over the leaves of the levels it
 * is given, modular_algorithm_assembler.cpp:957-988); leaf b's state is src[level]. */
static void glf_maxima_leaves(const Geom *g, const Eos *e, double *const *src, const int *level,
                              const int *items, int ni) {
  double m[3] = {0.0, 0.0, 0.0};
  double c[MAXNE], p[MAXNE];
  for (int n = 0; n < ni; ++n) {
    int const b = items[n];
    const double *ub = src[level[b]] + (long)b * g->ne * g->cells;
    for (int i = fic(g, 0); i <= lic(g, 0); ++i)
      for (int j = fic(g, 1); j <= lic(g, 1); ++j)
        for (int k = fic(g, 2); k <= lic(g, 2); ++k) {
          long const x = cidx(g, i, j, k);
          for (int f = 0; f < g->ne; ++f) c[f] = ub[f * g->cells + x];
          cons_to_prim(e, c, p);
          if (p[RHO] <= 0.0) continue;
          double const cs = eos_speed_of_sound(e, p[RHO], p[PRES]);
          double const vx = p[VELX];
          m[0] = dmax(m[0], fabs(vx - cs));
          m[1] = dmax(m[1], fabs(vx));
          m[2] = dmax(m[2], fabs(vx + cs));
        }
  }
  for (int q = 0; q < 3; ++q) g_glf[q] = m[q];
}

static int glf_selected(int solver) {
  return solver == ORACLE_FLUX_SPLITTING && g_splitting == FSP_GLF;
}

static void block_primes(const Geom *g, const Eos *e, const double *u, double *p) {
  double c[MAXNE], q[MAXNE];
  for (long x = 0; x < g->cells; ++x) {
    for (int f = 0; f < g->ne; ++f) c[f] = u[f * g->cells + x];
    cons_to_prim(e, c, q);
    for (int f = 0; f < g->np; ++f) p[f * g->cells + x] = q[f];
  }
}

/* face-index ranges of ComputeFluxes<DIR> (finite_volume_scheme.cpp:165-188) */
static void face_range(const Geom *g, int dir, int lo[3], int hi[3], int off[3]) {
  for (int d = 0; d < 3; ++d) {
    lo[d] = d == dir ? fic(g, d) - 1 : fic(g, d);
    hi[d] = lic(g, d);
    off[d] = d < g->dim ? fic(g, d) - 1 : -1;
  }
}

static void eigen_direction(const Geom *g, const Eos *e, int dir, const double *u,
                            const double *p, Eigen *eig) {
  int lo[3], hi[3], off[3];
  face_range(g, dir, lo, hi, off);
  for (int i = lo[0]; i <= hi[0]; ++i)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int k = lo[2]; k <= hi[2]; ++k) {
        long const t = cidx(g, i, j, k);
        long const n = cidx(g, i + (dir == 0), j + (dir == 1), k + (dir == 2));
        roe_eigen(g, e, dir, u, p, t, n, &eig[fidx(g, i - off[0], j - off[1], k - off[2])]);
      }
}

/* FiniteVolumeScheme::ComputeFluxes<DIR> (finite_volume_scheme.cpp:160-251) with
 * CharacteristicStateReconstruction (characteristic_state_reconstruction.h:57-136)
 * or PrimitiveStateReconstruction (primitive_state_reconstruction.h:56-107). */
static void fv_fluxes(const Geom *g, const Eos *e, int recon, int dir,
                      const double *u, const double *p, Eigen *eig, double *flux) {
  int const ne = g->ne, np = g->np;
  long const C = g->cells;
  int lo[3], hi[3], off[3];
  face_range(g, dir, lo, hi, off);
  int const *seq = summation_sequence(g->dim, dir);
  double const B = e->B;
  for (int i = lo[0]; i <= hi[0]; ++i)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int k = lo[2]; k <= hi[2]; ++k) {
        long const fi = fidx(g, i - off[0], j - off[1], k - off[2]);
        int const W = stencil_width(), D = W / 2 - 1;
        long cells6[MAXW];
        for (int m = 0; m < W; ++m) {
          int const s = m - D;
          cells6[m] = cidx(g, i + (dir == 0) * s, j + (dir == 1) * s, k + (dir == 2) * s);
        }
        double cm[MAXNE], cp[MAXNE], pm[MAXNE], pp[MAXNE];
        if (recon == ORACLE_RECON_CHARACTERISTIC) {
          double chm[MAXNE], chp[MAXNE], uc[MAXW];
          for (int n = 0; n < ne; ++n) {
            for (int m = 0; m < W; ++m) {
              uc[m] = 0.0;
              for (int s = 0; s < ne; ++s) {
                int const l = seq[s];
                uc[m] += eig[fi].L[n][l] * u[l * C + cells6[m]];
              }
            }
            chm[n] = recon_left(uc);
            chp[n] = recon_right(uc);
          }
          to_physical(ne, chm, eig[fi].R, cm);
          to_physical(ne, chp, eig[fi].R, cp);
          if (cm[MASS] <= DBL_EPSILON || cp[MASS] <= DBL_EPSILON) continue;
          cons_to_prim(e, cm, pm);
          cons_to_prim(e, cp, pp);
        } else {
          double arr[MAXW];
          for (int n = 0; n < np; ++n) {
            for (int m = 0; m < W; ++m) arr[m] = p[n * C + cells6[m]];
            pm[n] = recon_left(arr);
            pp[n] = recon_right(arr);
          }
          prim_to_cons(e, pm, cm);
          prim_to_cons(e, pp, cp);
        }
        if (cm[MASS] <= DBL_EPSILON || cp[MASS] <= DBL_EPSILON) continue;
        if (pm[PRES] <= -B || pp[PRES] <= -B) continue;
        double f[MAXNE];
        hllc(e, dir, cm, cp, pm, pp, f);
        for (int n = 0; n < ne; ++n) flux[n * g->faces + fi] += f[n];
      }
}

/* ComputeAdvection<DIR> (flux_splitting_scheme.cpp:42-76) */
static void advection(const Geom *g, int dir, const double *u, const double *p,
                      double *adv) {
  long const C = g->cells;
  for (long x = 0; x < C; ++x) {
    double const rho = p[RHO * C + x], pres = p[PRES * C + x];
    double const energy = u[ENERGY * C + x];
    double const vel = p[(VELX + dir) * C + x];
    adv[MASS * C + x] = rho * vel;
    adv[ENERGY * C + x] = (energy + pres) * vel;
    for (int d = 0; d < g->dim; ++d)
      adv[(MOMX + d) * C + x] = rho * (vel * p[(VELX + d) * C + x]);
    adv[(MOMX + dir) * C + x] += pres;
  }
}

/* FluxSplittingScheme::ComputeFluxes<DIR> (flux_splitting_scheme.cpp:185-315) */
static void fs_fluxes(const Geom *g, int dir, const double *u, const double *adv,
                      Eigen *eig, double *flux) {
  int const ne = g->ne;
  long const C = g->cells;
  int lo[3], hi[3], off[3];
  face_range(g, dir, lo, hi, off);
  int const *seq = summation_sequence(g->dim, dir);
  for (int i = lo[0]; i <= hi[0]; ++i)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int k = lo[2]; k <= hi[2]; ++k) {
        long const fi = fidx(g, i - off[0], j - off[1], k - off[2]);
        int const W = stencil_width(), D = W / 2 - 1;
        long cells6[MAXW];
        for (int m = 0; m < W; ++m) {
          int const s = m - D;
          cells6[m] = cidx(g, i + (dir == 0) * s, j + (dir == 1) * s, k + (dir == 2) * s);
        }
        double chf[MAXNE], pos[MAXW], neg[MAXW], phys[MAXNE];
        for (int n = 0; n < ne; ++n) {
          double const alpha = eig[fi].ev[n];
          for (int m = 0; m < W; ++m) {
            pos[m] = 0.0;
            neg[m] = 0.0;
            for (int s = 0; s < ne; ++s) {
              int const l = seq[s];
              double const uct = u[l * C + cells6[m]] * eig[fi].L[n][l];
              double const act = adv[l * C + cells6[m]] * eig[fi].L[n][l];
              pos[m] += (act + alpha * uct);
              neg[m] += (act - alpha * uct);
            }
          }
          chf[n] = 0.5 * (recon_left(pos) + recon_right(neg));
        }
        to_physical(ne, chf, eig[fi].R, phys);
        for (int l = 0; l < ne; ++l) flux[l * g->faces + fi] += phys[l];
      }
}

/* Convective fluxes of one block (FiniteVolumeScheme::UpdateImplementation,
 * finite_volume_scheme.cpp:45-145; FluxSplittingScheme::UpdateImplementation,
 * flux_splitting_scheme.cpp:97-168). fx, fy, fz are zeroed first as
 * SpaceSolver::UpdateFluxes does (space_solver.cpp:89-98). */
static void block_fluxes(const Geom *g, const Eos *e, int solver, int recon,
                         const double *u, Work *w, double *f[3]) {
  long const nf = (long)g->ne * g->faces;
  for (int d = 0; d < 3; ++d) memset(f[d], 0, sizeof(double) * nf);
  block_primes(g, e, u, w->prim);
  memset(w->eig, 0, sizeof(Eigen) * g->faces);
  int const need_eigen = solver == ORACLE_FLUX_SPLITTING ||
                         recon == ORACLE_RECON_CHARACTERISTIC;
  for (int dir = 0; dir < g->dim; ++dir) {
    if (need_eigen) eigen_direction(g, e, dir, u, w->prim, w->eig);
    if (solver == ORACLE_FINITE_VOLUME) {
      fv_fluxes(g, e, recon, dir, u, w->prim, w->eig, f[dir]);
    } else {
      advection(g, dir, u, w->prim, w->adv);
      fs_fluxes(g, dir, u, w->adv, w->eig, f[dir]);
    }
  }
}

/* RHS zeroing and divergence of SpaceSolver::UpdateFluxes
 * (space_solver.cpp:58-70, 131-153); volume forces are zero. */
static void block_divergence(const Geom *g, double cell_size, double *f[3],
                             double *rhs) {
  memset(rhs, 0, sizeof(double) * g->ne * g->cells);
  double const one_cell_size = 1.0 / cell_size;
  for (int e = 0; e < g->ne; ++e) {
    const double *fx = f[0] + e * g->faces;
    const double *fy = f[1] + e * g->faces;
    const double *fz = f[2] + e * g->faces;
    for (int i = 0; i < g->ic[0]; ++i)
      for (int j = 0; j < g->ic[1]; ++j)
        for (int k = 0; k < g->ic[2]; ++k) {
          double const dx = fx[fidx(g, i, j + 1, k + 1)] - fx[fidx(g, i + 1, j + 1, k + 1)];
          double const dy = fy[fidx(g, i + 1, j, k + 1)] - fy[fidx(g, i + 1, j + 1, k + 1)];
          double const dz = fz[fidx(g, i + 1, j + 1, k)] - fz[fidx(g, i + 1, j + 1, k + 1)];
          long const c = cidx(g, i + fic(g, 0), j + fic(g, 1), k + fic(g, 2));
          rhs[e * g->cells + c] += 0.0 + dacms(g->dim, dx, dy, dz) * one_cell_size;
        }
  }
}

/* ---- threading ---------------------------------------------------------- */

typedef void (*task_fn)(void *ctx, int block, Work *w, double *f[3]);
typedef struct {
  task_fn fn;
  void *ctx;
  const Geom *g;
  int nb, nthreads, tid;
} ThreadArg;

static void *thread_main(void *p) {
  ThreadArg *a = (ThreadArg *)p;
  Work w;
  work_alloc(a->g, &w);
  long const nf = (long)a->g->ne * a->g->faces;
  double *fb = (double *)malloc(sizeof(double) * 3 * nf);
  double *f[3] = {fb, fb + nf, fb + 2 * nf};
  for (int b = a->tid; b < a->nb; b += a->nthreads) a->fn(a->ctx, b, &w, f);
  free(fb);
  work_free(&w);
  return NULL;
}

static void parallel_blocks(const Geom *g, int nb, int nthreads, task_fn fn, void *ctx) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > nb) nthreads = nb > 0 ? nb : 1;
  pthread_t th[256];
  ThreadArg args[256];
  if (nthreads > 256) nthreads = 256;
  for (int t = 0; t < nthreads; ++t) {
    args[t].fn = fn;
    args[t].ctx = ctx;
    args[t].g = g;
    args[t].nb = nb;
    args[t].nthreads = nthreads;
    args[t].tid = t;
  }
  if (nthreads == 1) {
    thread_main(&args[0]);
    return;
  }
  for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, thread_main, &args[t]);
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
}

/* ---- public entry points ------------------------------------------------ */

int oracle_weno5(const double *v6, double *left, double *right) {
  *left = weno5_left(v6);
  *right = weno5_right(v6);
  return 0;
}

int oracle_eos(int dim, double gamma, double B, int safe, const double *cons,
               const double *prim, double *out) {
  Eos e = {dim, gamma, B, safe};
  out[0] = eos_pressure(&e, cons[0], cons[2], cons[3], cons[4], cons[1]);
  out[1] = eos_enthalpy(&e, cons[0], cons[2], cons[3], cons[4], cons[1]);
  out[2] = eos_energy(&e, prim[0], prim[2], prim[3], prim[4], prim[1]);
  out[3] = eos_speed_of_sound(&e, prim[0], prim[1]);
  out[4] = eos_psi(&e, prim[1], 1.0 / prim[0]);
  out[5] = eos_gruneisen(&e);
  return 0;
}

int oracle_prime_states(int dim, const double *u, int nb, double gamma, double B,
                        int safe, double *p) {
  if (dim < 1 || dim > 3) return 1;
  Geom g = make_geom(dim);
  Eos e = {dim, gamma, B, safe};
  for (int b = 0; b < nb; ++b)
    block_primes(&g, &e, u + (long)b * g.ne * g.cells, p + (long)b * g.np * g.cells);
  return 0;
}

typedef struct {
  const Geom *g;
  const Eos *e;
  int solver, recon;
  const double *u;
  double cell_size;
  double *fx, *fy, *fz, *rhs;
} RhsCtx;

static void rhs_task(void *vctx, int b, Work *w, double *f[3]) {
  RhsCtx *c = (RhsCtx *)vctx;
  const Geom *g = c->g;
  long const nf = (long)g->ne * g->faces;
  block_fluxes(g, c->e, c->solver, c->recon, c->u + (long)b * g->ne * g->cells, w, f);
  if (c->fx) memcpy(c->fx + b * nf, f[0], sizeof(double) * nf);
  if (c->fy) memcpy(c->fy + b * nf, f[1], sizeof(double) * nf);
  if (c->fz) memcpy(c->fz + b * nf, f[2], sizeof(double) * nf);
  if (c->rhs) block_divergence(g, c->cell_size, f, c->rhs + (long)b * g->ne * g->cells);
}

int oracle_space_rhs(int dim, int solver, int recon, const double *u, int nb,
                     double gamma, double B, int safe, double cell_size, double *fx,
                     double *fy, double *fz, double *rhs, int nthreads) {
  if (dim < 1 || dim > 3) return 1;
  if (solver == ORACLE_FINITE_VOLUME && recon == ORACLE_RECON_CONSERVATIVE) return 2;
  Geom g = make_geom(dim);
  Eos e = {dim, gamma, B, safe};
  RhsCtx c = {&g, &e, solver, recon, u, cell_size, fx, fy, fz, rhs};
  if (glf_selected(solver)) glf_maxima(&g, &e, u, nb);
  parallel_blocks(&g, nb, nthreads, rhs_task, &c);
  return 0;
}

/* ComputeTimestepSize (modular_algorithm_assembler.cpp:1840-1870, 1932,
 * 1961-1982): max over interior cells of the consistency-managed sum of
 * |u_d| + c, dt = CFL / (s / dx), clipped to the end time. The zero
 * viscous / capillary / heat / gravity max() terms leave dt unchanged. */
int oracle_timestep(int dim, const double *u, int nb, double gamma, double B,
                    int safe, double cell_size, double cfl, double t, double t_end,
                    double *dt_out) {
  Geom g = make_geom(dim);
  Eos e = {dim, gamma, B, safe};
  double s = 0.0;
  double c[MAXNE], p[MAXNE], vps[3];
  for (int b = 0; b < nb; ++b) {
    const double *ub = u + (long)b * g.ne * g.cells;
    for (int i = fic(&g, 0); i <= lic(&g, 0); ++i)
      for (int j = fic(&g, 1); j <= lic(&g, 1); ++j)
        for (int k = fic(&g, 2); k <= lic(&g, 2); ++k) {
          long const x = cidx(&g, i, j, k);
          for (int f = 0; f < g.ne; ++f) c[f] = ub[f * g.cells + x];
          cons_to_prim(&e, c, p);
          double const cs = eos_speed_of_sound(&e, p[RHO], p[PRES]);
          for (int d = 0; d < dim; ++d) vps[d] = fabs(p[VELX + d]) + cs;
          s = dmax(s, cms_array(dim, vps));
        }
  }
  double dt = s / cell_size;
  double local;
  if (dt == 0.0)
    local = DBL_MAX;
  else
    local = cfl / dt;
  if (t + local > t_end) local = dmax(t_end - t, 0.0);
  *dt_out = local;
  return 0;
}

/* Zero-gradient slabs of the domain faces (boundary_constants.h:103-160,
 * 211-252): the full TCY x TCZ (etc.) halo slab takes the first / last
 * interior plane. A face is a domain face when face_nbr(b, face) < 0. */
/* A neighbour entry of -2 marks a symmetry wall instead
 * (symmetry_boundary_condition.h:60-113, boundary_constants.h:35-46, 167-209):
 * the halo cell at distance q from the wall takes the interior cell at
 * distance q on the other side, the momentum normal to the wall negated
 * (SymmetrySign -1.0, symmetry_boundary_condition.h:148-217). */
static void zero_gradient_slabs(const Geom *g, double *u, int nb, int nfields,
                                const int *nbr, int nbr_stride, const int *face_slot) {
  for (int b = 0; b < nb; ++b)
    for (int face = 0; face < 2 * g->dim; ++face) {
      int const nb_face = nbr[(long)nbr_stride * b + face_slot[face]];
      if (nb_face >= 0) continue;
      int const sym = nb_face == -2;
      int const dir = face / 2, high = face % 2;
      int const s = high ? HS + IC - 1 : HS;
      int const mirror = high ? 2 * (HS + IC) - 1 : 2 * HS - 1;
      int const h0 = high ? HS + IC : 0, h1 = high ? TC : HS;
      for (int f = 0; f < nfields; ++f) {
        double *x = u + ((long)b * nfields + f) * g->cells;
        double const sign = (sym && f == MOMX + dir) ? -1.0 : 1.0;
        for (int i = 0; i < g->tc[0]; ++i)
          for (int j = 0; j < g->tc[1]; ++j)
            for (int k = 0; k < g->tc[2]; ++k) {
              int const idx[3] = {i, j, k};
              if (idx[dir] < h0 || idx[dir] >= h1) continue;
              int si = i, sj = j, sk = k;
              int const src = sym ? mirror - idx[dir] : s;
              if (dir == 0) si = src;
              if (dir == 1) sj = src;
              if (dir == 2) sk = src;
              x[cidx(g, i, j, k)] = sym ? sign * x[cidx(g, si, sj, sk)] : x[cidx(g, si, sj, sk)];
            }
      }
    }
}

/* slot of face W,E,S,N,B,T in the 26-entry table */
static const int face_slot26[6] = {4, 21, 10, 15, 12, 13};
static const int face_slot6[6] = {0, 1, 2, 3, 4, 5};

/* Same-level halo copy. nbr26 holds 26 neighbour indices per block (-1: none),
 * ordered by direction offsets (ox, oy, oz) in {-1,0,1}^3 \ {0} with ox slowest:
 * index = (ox+1)*9 + (oy+1)*3 + (oz+1), minus one past the centre (13). The
 * region for offset +1 is [HS+IC, TC) filled from the neighbour's [HS, 2HS),
 * for -1 it is [0, HS) from the neighbour's [IC, IC+HS), for 0 the interior
 * (communication_types.h:45-132; internal_halo_manager.cpp:439-459).
 * faces_only copies only the 2*dim planes; zero_gradient then applies the
 * domain-face slabs, external after internal as in halo_manager.cpp:87-124. */
int oracle_halo_fill(int dim, double *u, int nb, int nfields, const int *nbr26,
                     int faces_only, int zero_gradient) {
  Geom g = make_geom(dim);
  for (int b = 0; b < nb; ++b) {
    for (int o = 0; o < 27; ++o) {
      if (o == 13) continue;
      int const oo[3] = {o / 9 - 1, (o / 3) % 3 - 1, o % 3 - 1};
      int nz = 0, skip = 0;
      for (int d = 0; d < 3; ++d) {
        if (oo[d] != 0) ++nz;
        if (d >= dim && oo[d] != 0) skip = 1;
      }
      if (skip || (faces_only && nz != 1)) continue;
      int const slot = o < 13 ? o : o - 1;
      int const n = nbr26[26 * b + slot];
      if (n < 0) continue;
      int lo[3], ext[3], src[3];
      for (int d = 0; d < 3; ++d) {
        if (d >= dim) {
          lo[d] = 0; ext[d] = 1; src[d] = 0;
        } else if (oo[d] == 0) {
          lo[d] = HS; ext[d] = IC; src[d] = HS;
        } else if (oo[d] > 0) {
          lo[d] = HS + IC; ext[d] = HS; src[d] = HS;
        } else {
          lo[d] = 0; ext[d] = HS; src[d] = IC;
        }
      }
      for (int f = 0; f < nfields; ++f) {
        double *dst = u + ((long)b * nfields + f) * g.cells;
        const double *s = u + ((long)n * nfields + f) * g.cells;
        for (int i = 0; i < ext[0]; ++i)
          for (int j = 0; j < ext[1]; ++j)
            for (int k = 0; k < ext[2]; ++k)
              dst[cidx(&g, lo[0] + i, lo[1] + j, lo[2] + k)] =
                  s[cidx(&g, src[0] + i, src[1] + j, src[2] + k)];
      }
    }
  }
  if (zero_gradient) zero_gradient_slabs(&g, u, nb, nfields, nbr26, 26, face_slot26);
  return 0;
}

/* Face halos from the six-entry neighbour table (W,E,S,N,B,T) followed by the
 * zero-gradient slabs of domain faces (boundary_constants.h:103-160, 211-252),
 * external after internal as in halo_manager.cpp:87-124. */
static void halo_update6(const Geom *g, double *u, int nb, const int *nbr) {
  int const ne = g->ne;
  for (int b = 0; b < nb; ++b)
    for (int face = 0; face < 2 * g->dim; ++face) {
      int const n = nbr[6 * b + face];
      if (n < 0) continue;
      int const dir = face / 2, high = face % 2;
      int lo[3], ext[3], src[3];
      for (int d = 0; d < 3; ++d) {
        lo[d] = fic(g, d);
        ext[d] = g->ic[d];
        src[d] = fic(g, d);
      }
      ext[dir] = HS;
      lo[dir] = high ? HS + IC : 0;
      src[dir] = high ? HS : IC;
      for (int f = 0; f < ne; ++f) {
        double *dst = u + ((long)b * ne + f) * g->cells;
        const double *s = u + ((long)n * ne + f) * g->cells;
        for (int i = 0; i < ext[0]; ++i)
          for (int j = 0; j < ext[1]; ++j)
            for (int k = 0; k < ext[2]; ++k)
              dst[cidx(g, lo[0] + i, lo[1] + j, lo[2] + k)] =
                  s[cidx(g, src[0] + i, src[1] + j, src[2] + k)];
      }
    }
  zero_gradient_slabs(g, u, nb, ne, nbr, 6, face_slot6);
}

int oracle_halo_update(int dim, double *u, int nb, const int *nbr) {
  if (dim < 1 || dim > 3) return 1;
  Geom g = make_geom(dim);
  halo_update6(&g, u, nb, nbr);
  return 0;
}

/* SSP-RK3 (runge_kutta_3_TVD.h:41-59) and TVD-RK2 (runge_kutta_2_TVD.h:37-56):
 * per stage the multiplier of dt and the buffer multipliers of the stage input
 * and of the step's initial state; the integrator is selected at run time
 * (TimeIntegrators of numerical_setup.h: RK2 = 0, RK3 = 1). */
enum { TI_RK2 = 0, TI_RK3 = 1 };
static int g_integrator = TI_RK3;
static const double rk3_c[3] = {1.0, 0.25, 2.0 / 3.0};
static const double rk3_a[3][2] = {{0.0, 0.0}, {0.25, 0.75}, {2.0 / 3.0, 1.0 / 3.0}};
static const double rk2_c[3] = {1.0, 0.5, 0.0};
static const double rk2_a[3][2] = {{0.0, 0.0}, {0.5, 0.5}, {0.0, 0.0}};
static int rk_stages(void) { return g_integrator == TI_RK2 ? 2 : 3; }

int oracle_set_time_integrator(int integrator) {
  if (integrator != TI_RK2 && integrator != TI_RK3) return 1;
  g_integrator = integrator;
  return 0;
}

typedef struct {
  const Geom *g;
  const Eos *e;
  int solver, recon, stage;
  double *u, *u0, *rhs;
  double cell_size, dt;
} StageCtx;

/* ComputeRightHandSide per block (modular_algorithm_assembler.cpp:990-1007):
 * FillInitialBuffer (time_integrator.h:369-406), UpdateFluxes, then
 * PrepareBufferForIntegration (time_integrator.h:434-457) over all cells, then
 * IntegrateConservatives (time_integrator.h:98-113) on the interior. */
static void stage_task(void *vctx, int b, Work *w, double *f[3]) {
  StageCtx *c = (StageCtx *)vctx;
  const Geom *g = c->g;
  long const n = (long)g->ne * g->cells;
  double *u = c->u + b * n, *u0 = c->u0 + b * n, *r = c->rhs + b * n;
  if (c->stage == 0) memcpy(u0, u, sizeof(double) * n);
  block_fluxes(g, c->e, c->solver, c->recon, u, w, f);
  block_divergence(g, c->cell_size, f, r);
  const double(*rka)[2] = g_integrator == TI_RK2 ? rk2_a : rk3_a;
  const double *const rkc = g_integrator == TI_RK2 ? rk2_c : rk3_c;
  if (c->stage != 0) {
    double const m0 = rka[c->stage][0], m1 = rka[c->stage][1];
    for (long x = 0; x < n; ++x) u[x] = m0 * u[x] + m1 * u0[x];
  }
  double const step = rkc[c->stage] * (0.0 + c->dt);
  for (int e = 0; e < g->ne; ++e)
    for (int i = fic(g, 0); i <= lic(g, 0); ++i)
      for (int j = fic(g, 1); j <= lic(g, 1); ++j)
        for (int k = fic(g, 2); k <= lic(g, 2); ++k) {
          long const x = e * g->cells + cidx(g, i, j, k);
          r[x] = u[x] + step * r[x];
        }
}

/* Single-level, single-phase Advance (modular_algorithm_assembler.cpp:575-874):
 * dt, then three stages of RHS / prepare / integrate, halo update of the
 * integrated buffer (:726) and the buffer swap (:830). */
int oracle_run(int dim, int solver, int recon, double *u, int nb, const int *nbr,
               double gamma, double B, int safe, double cell_size, double cfl,
               double t_end, int max_steps, int nthreads, double *t_io,
               int *steps_done, double *dt_log) {
  if (dim < 1 || dim > 3) return 1;
  Geom g = make_geom(dim);
  Eos e = {dim, gamma, B, safe};
  long const n = (long)nb * g.ne * g.cells;
  double *u0 = (double *)malloc(sizeof(double) * n);
  double *rhs = (double *)malloc(sizeof(double) * n);
  if (!u0 || !rhs) {
    free(u0);
    free(rhs);
    return 3;
  }
  memcpy(u0, u, sizeof(double) * n);
  memcpy(rhs, u, sizeof(double) * n);
  halo_update6(&g, u, nb, nbr);
  double *cur = u, *other = rhs;
  double t = *t_io;
  int steps = 0;
  while (t < t_end && (max_steps <= 0 || steps < max_steps)) {
    double dt;
    oracle_timestep(dim, cur, nb, gamma, B, safe, cell_size, cfl, t, t_end, &dt);
    if (dt_log) dt_log[steps] = dt;
    for (int stage = 0; stage < rk_stages(); ++stage) {
      StageCtx c = {&g, &e, solver, recon, stage, cur, u0, other, cell_size, dt};
      if (glf_selected(solver)) glf_maxima(&g, &e, cur, nb);
      parallel_blocks(&g, nb, nthreads, stage_task, &c);
      halo_update6(&g, other, nb, nbr);
      double *tmp = cur;
      cur = other;
      other = tmp;
    }
    t = t + (0.0 + dt);
    ++steps;
  }
  if (cur != u) memcpy(u, cur, sizeof(double) * n);
  free(u0);
  free(rhs);
  *t_io = t;
  *steps_done = steps;
  return 0;
}

/* ---- multi-level cases: a block tree with local time stepping ------------
 *
 * Leaves of levels 0..lmax tile a box of n0[0] x n0[1] x n0[2] level-0 nodes
 * (inactive dimensions 1); a node of level l has cell size h0 / 2^l and
 * integer coordinates in units of its own size. Time stepping restates
 * ModularAlgorithmAssembler::Advance (modular_algorithm_assembler.cpp:575-874):
 * a macro step is 2^lmax micro steps; micro step t integrates the levels of
 * GetLevels(t) (:2564-2573), level l with the sum of its last 2^(lmax-l) micro
 * time steps (Integrate :1068-1098, time_integrator.h:312-340); the stage-0
 * right-hand side of a level is evaluated at the start of its interval
 * (levels of GetLevels(t-1), all levels at t = 0). The micro time step is
 * ComputeTimestepSize over all leaves with the finest cell size, clipped to
 * the end time with the micro steps taken so far (:1925-1982); the macro time
 * advances by their sum (FinishMacroTimestep, time_integrator.h:247-252).
 * A level whose time step is zero is not integrated.
 *
 * Halo cells across a jump (a face neighbour one level coarser or finer) are
 * filled by averaging the finer leaves with Multiresolution::Average
 * (multiresolution.h:94-166) and, on the finer side, by the fifth-order
 * prediction from the coarser level (Multiresolution::Prediction,
 * multiresolution.cpp:146-283), through the level field below.
 * Conservation at jumps follows the reference: every leaf integrates its
 * boundary face fluxes at jump faces with the RK3 jump multipliers (1/6, 1/6,
 * 2/3) times its level step (SpaceSolver::UpdateFluxes space_solver.cpp:155-182,
 * IntegrateJumpConservatives time_integrator.h:64-80, runge_kutta_3_TVD.h:42-46);
 * at the end of each fine step these sums are averaged onto the parent's face
 * (Multiresolution::AverageJumpBuffer, multiresolution.cpp:47-128) and reset;
 * at the end of a coarse step the cells of a coarse leaf next to a refined
 * neighbour get - CMS(coarse sums) + CMS(fine sums) per unit cell size
 * (JumpFluxAdjustment, modular_algorithm_assembler.cpp:1347-1636) and the sums
 * are reset. Face neighbours must differ by at most one level.
 */

#define MAXLEV 8

typedef struct {
  int dim, lmax, nleaf;
  int ext[MAXLEV][3];
  int *grid[MAXLEV]; /* >= 0 leaf index, -1 inside a coarser leaf, -2 refined */
  const int *level, *coord;
} Tree;

static long tree_at(const Tree *t, int l, const int c[3]) {
  return ((long)c[0] * t->ext[l][1] + c[1]) * t->ext[l][2] + c[2];
}

static void tree_free(Tree *t) {
  for (int l = 0; l < MAXLEV; ++l) free(t->grid[l]);
}

/* 0 ok, 4 not a tiling of the box, 5 face neighbours more than one level apart */
static int tree_build(Tree *t, int dim, int nleaf, const int *level, const int *coord,
                      const int *n0) {
  memset(t, 0, sizeof(*t));
  t->dim = dim;
  t->nleaf = nleaf;
  t->level = level;
  t->coord = coord;
  int lmax = 0;
  for (int b = 0; b < nleaf; ++b) {
    if (level[b] < 0 || level[b] >= MAXLEV) return 4;
    if (level[b] > lmax) lmax = level[b];
  }
  t->lmax = lmax;
  for (int l = 0; l <= lmax; ++l) {
    long n = 1;
    for (int d = 0; d < 3; ++d) {
      t->ext[l][d] = d < dim ? n0[d] << l : 1;
      n *= t->ext[l][d];
    }
    t->grid[l] = (int *)malloc(sizeof(int) * n);
    if (!t->grid[l]) return 3;
    for (long x = 0; x < n; ++x) t->grid[l][x] = -1;
  }
  for (int b = 0; b < nleaf; ++b) {
    int const l = level[b];
    int c[3];
    for (int d = 0; d < 3; ++d) {
      c[d] = d < dim ? coord[3 * b + d] : 0;
      if (c[d] < 0 || c[d] >= t->ext[l][d]) return 4;
    }
    long const x = tree_at(t, l, c);
    if (t->grid[l][x] != -1) return 4;
    t->grid[l][x] = b;
  }
  for (int b = 0; b < nleaf; ++b)
    for (int a = level[b] - 1; a >= 0; --a) {
      int c[3];
      for (int d = 0; d < 3; ++d) c[d] = d < dim ? coord[3 * b + d] >> (level[b] - a) : 0;
      long const x = tree_at(t, a, c);
      if (t->grid[a][x] >= 0) return 4;
      t->grid[a][x] = -2;
    }
  /* every level-0 node present, every refined node has all its children */
  for (int l = 0; l <= lmax; ++l) {
    for (int i = 0; i < t->ext[l][0]; ++i)
      for (int j = 0; j < t->ext[l][1]; ++j)
        for (int k = 0; k < t->ext[l][2]; ++k) {
          int const c[3] = {i, j, k};
          int const v = t->grid[l][tree_at(t, l, c)];
          if (l == 0 && v == -1) return 4;
          if (v == -2) {
            if (l == lmax) return 4;
            for (int o = 0; o < (1 << dim); ++o) {
              int cc[3];
              for (int d = 0; d < 3; ++d) cc[d] = d < dim ? 2 * c[d] + ((o >> d) & 1) : 0;
              if (t->grid[l + 1][tree_at(t, l + 1, cc)] == -1) return 4;
            }
          }
        }
  }
  /* face balance: the neighbour region of a leaf is a leaf of its level, a
   * refined node whose face children are leaves, or lies in a leaf one level
   * coarser */
  for (int b = 0; b < nleaf; ++b) {
    int const l = level[b];
    for (int f = 0; f < 2 * dim; ++f) {
      int const d = f / 2, s = (f % 2) ? 1 : -1;
      int p[3];
      for (int e = 0; e < 3; ++e) p[e] = e < dim ? coord[3 * b + e] : 0;
      p[d] += s;
      if (p[d] < 0 || p[d] >= t->ext[l][d]) continue;
      int const v = t->grid[l][tree_at(t, l, p)];
      if (v == -1) {
        int q[3];
        for (int e = 0; e < 3; ++e) q[e] = e < dim ? p[e] >> 1 : 0;
        if (l == 0 || t->grid[l - 1][tree_at(t, l - 1, q)] < 0) return 5;
      } else if (v == -2) {
        for (int o = 0; o < (1 << dim); ++o) {
          if (((o >> d) & 1) != (s > 0 ? 0 : 1)) continue;
          int cc[3];
          for (int e = 0; e < 3; ++e) cc[e] = e < dim ? 2 * p[e] + ((o >> e) & 1) : 0;
          if (t->grid[l + 1][tree_at(t, l + 1, cc)] < 0) return 5;
        }
      }
    }
  }
  return 0;
}

/* 3D / 2D / 1D conservative average of the 2^dim children cells of a parent
 * cell (Multiresolution::Average, multiresolution.h:133-158). c points at the
 * child cell (2a, 2b, 2c) of field buffer f. */
/* w[o]: child o (bit d of o: high half along d) */
static double average_values(int dim, const double *w) {
  if (dim == 1) return (w[0] + w[1]) * 0.5;
  if (dim == 2) return ((w[0] + w[3]) + (w[1] + w[2])) * 0.25;
  double const a = w[0] + w[7];
  double const b = w[4] + w[3];
  double const c = w[2] + w[5];
  double const d = w[6] + w[1];
  double const s1 = (a + b) + (c + d);
  double const s2 = (a + c) + (b + d);
  double const s3 = (a + d) + (b + c);
  double const mn = dmin(s1, dmin(s2, s3)), mx = dmax(s1, dmax(s2, s3));
  return 0.125 * (0.5 * (mn + mx));
}

static double child_average(const Geom *g, const double *f, int i, int j, int k) {
  double w[8];
  for (int o = 0; o < (1 << g->dim); ++o)
    w[o] = f[cidx(g, i + (o & 1), j + ((o >> 1) & 1), k + ((o >> 2) & 1))];
  return average_values(g->dim, w);
}

/* ConsistencyManagedSum of four values (mathematical_functions.h:115-125) */
static double cms4(double a, double b, double c, double d) {
  double const s1 = (a + b) + (c + d);
  double const s2 = (a + c) + (b + d);
  double const s3 = (a + d) + (b + c);
  double mn = s1, mx = s1;
  if (s2 < mn) mn = s2;
  if (s3 < mn) mn = s3;
  if (mx < s2) mx = s2;
  if (mx < s3) mx = s3;
  return 0.5 * (mn + mx);
}

/* Fifth-order prediction of the children of one parent cell
 * (Multiresolution::Prediction, multiresolution.cpp:146-283, after Harten 1993).
 * v: the parent values at offsets -2..2 around the cell, v[(a+2)*25 + (b+2)*5 +
 * (c+2)] for offsets (a, b, c) along x, y, z (offsets of absent dimensions 0).
 * out[o]: child o, bit d of o set for the high-index child along d. The terms
 * and their evaluation order are the reference's: differences along one axis
 * (Qx, Qy, Qz), pairs of axes (Qxy, Qxz, Qyz) and the consistency-managed
 * triple term (Qxyz), combined per child with the child's signs. */
#define PRED_V(a, b, c) v[((a) + 2) * 25 + ((b) + 2) * 5 + ((c) + 2)]
static const double pc0 = -22.0 / 128.0, pc1 = 3.0 / 128.0;

/* value at offset s along dimension d */
static double pred_at1(const double *v, int d, int s) {
  int o[3] = {0, 0, 0};
  o[d] = s;
  return PRED_V(o[0], o[1], o[2]);
}

/* value at offsets s along d and t along e */
static double pred_at2(const double *v, int d, int s, int e, int t) {
  int o[3] = {0, 0, 0};
  o[d] = s;
  o[e] = t;
  return PRED_V(o[0], o[1], o[2]);
}

static double pred_q1(const double *v, int d) {
  return pc0 * (pred_at1(v, d, 1) - pred_at1(v, d, -1)) +
         pc1 * (pred_at1(v, d, 2) - pred_at1(v, d, -2));
}

/* one coefficient's cross difference: (v(+a,+b) + v(-a,-b)) - (v(-a,+b) + v(+a,-b)) */
static double pred_x2(const double *v, int d, int e, int a, int b) {
  return (pred_at2(v, d, a, e, b) + pred_at2(v, d, -a, e, -b)) -
         (pred_at2(v, d, -a, e, b) + pred_at2(v, d, a, e, -b));
}

static double pred_q2(const double *v, int d, int e) {
  double const c00 = pc0 * pc0, c01 = pc0 * pc1, c11 = pc1 * pc1;
  return (c00 * pred_x2(v, d, e, 1, 1) + c11 * pred_x2(v, d, e, 2, 2)) +
         (c01 * pred_x2(v, d, e, 1, 2) + c01 * pred_x2(v, d, e, 2, 1));
}

/* the four antisymmetric differences of offsets (a, b, c), summed consistently */
static double pred_x3(const double *v, int a, int b, int c) {
  return cms4(PRED_V(a, b, c) - PRED_V(-a, -b, -c), PRED_V(-a, -b, c) - PRED_V(a, b, -c),
              PRED_V(a, -b, -c) - PRED_V(-a, b, c), PRED_V(-a, b, -c) - PRED_V(a, -b, c));
}

static double pred_q3(const double *v) {
  double const c00 = pc0 * pc0, c11 = pc1 * pc1;
  double const c000 = c00 * pc0, c001 = c00 * pc1, c011 = pc0 * c11, c111 = pc1 * c11;
  return cms4(c000 * pred_x3(v, 1, 1, 1) + c111 * pred_x3(v, 2, 2, 2),
              c001 * pred_x3(v, 1, 1, 2) + c011 * pred_x3(v, 2, 2, 1),
              c011 * pred_x3(v, 1, 2, 2) + c001 * pred_x3(v, 2, 1, 1),
              c001 * pred_x3(v, 1, 2, 1) + c011 * pred_x3(v, 2, 1, 2));
}

static void predict_children(int dim, const double *v, double out[8]) {
  double qx = 0.0, qy = 0.0, qz = 0.0, qxy = 0.0, qxz = 0.0, qyz = 0.0, qxyz = 0.0;
  qx = pred_q1(v, 0);
  if (dim > 1) {
    qy = pred_q1(v, 1);
    qxy = pred_q2(v, 0, 1);
  }
  if (dim > 2) {
    qz = pred_q1(v, 2);
    qxz = pred_q2(v, 0, 2);
    qyz = pred_q2(v, 1, 2);
    qxyz = pred_q3(v);
  }
  double const p = PRED_V(0, 0, 0);
  for (int o = 0; o < (1 << dim); ++o) {
    double const sx = (o & 1) ? -1.0 : 1.0, sy = (o & 2) ? -1.0 : 1.0, sz = (o & 4) ? -1.0 : 1.0;
    out[o] = p + dacms(dim, sx * qx, sy * qy, sz * qz) +
             dacms(dim, sx * sy * qxy, sx * sz * qxz, sy * sz * qyz) + sx * sy * sz * qxyz;
  }
}

/* Multiresolution::Prediction over a cell range of one field buffer: parent
 * and child are [tc] buffers of one field; the child has position octant among
 * its siblings; start / count give the child cells to fill (start even). */
int oracle_prediction(int dim, const double *parent, int octant, const int *start,
                      const int *count, double *child) {
  if (dim < 1 || dim > 3) return 1;
  Geom const gg = make_geom(dim);
  Geom const *g = &gg;
  int ps[3], pn[3];
  for (int d = 0; d < 3; ++d) {
    if (d < dim && (start[d] % 2 || count[d] % 2)) return 1;
    int const off = ((octant >> d) & 1) ? g->tc[0] / 2 - HS / 2 : HS / 2;
    ps[d] = d < dim ? start[d] / 2 + off : 0;
    pn[d] = d < dim ? count[d] / 2 : 1;
  }
  double v[125];
  for (int i = 0; i < pn[0]; ++i)
    for (int j = 0; j < pn[1]; ++j)
      for (int k = 0; k < pn[2]; ++k) {
        int const c[3] = {ps[0] + i, ps[1] + j, ps[2] + k};
        for (int a = -2; a <= 2; ++a)
          for (int b = -2; b <= 2; ++b)
            for (int e = -2; e <= 2; ++e) {
              int const q[3] = {c[0] + a, c[1] + (dim > 1 ? b : 0), c[2] + (dim > 2 ? e : 0)};
              int inside = 1;
              for (int d = 0; d < dim; ++d) inside &= q[d] >= 0 && q[d] < g->tc[d];
              PRED_V(a, b, e) = inside ? parent[cidx(g, q[0], q[1], q[2])] : 0.0;
            }
        double out[8];
        predict_children(dim, v, out);
        for (int o = 0; o < (1 << dim); ++o) {
          int x[3] = {0, 0, 0};
          for (int d = 0; d < dim; ++d) x[d] = start[d] + 2 * (d == 0 ? i : d == 1 ? j : k) + ((o >> d) & 1);
          child[cidx(g, x[0], x[1], x[2])] = out[o];
        }
      }
  return 0;
}

/* The cell values a node buffer of level L holds in the reference, for every
 * node position of level L: a leaf's own cells; a refined node's interior is
 * the average of its children (Averager, Multiresolution::Average); a node
 * position inside a coarser leaf is what a node there receives in its jump
 * halos, the prediction from the next coarser level (Multiresolution::
 * Prediction from the parent's buffer, internal_halo_manager.cpp:230-290);
 * beyond the domain, the zero-gradient value of the nearest domain cell. Refined
 * and predicted nodes are computed whole on first use and kept for the pass
 * (the leaves' values come from src[level], fixed during a pass). */
typedef struct {
  const Geom *g;
  const Tree *t;
  double *const *src;
  double **node[MAXLEV]; /* per level and node position: NULL or [ne][IC^dim] */
} LevelField;

static void lf_init(LevelField *F, const Geom *g, const Tree *t, double *const *src) {
  memset(F, 0, sizeof(*F));
  F->g = g;
  F->t = t;
  F->src = src;
}

static void lf_free(LevelField *F) {
  for (int l = 0; l < MAXLEV; ++l) {
    if (!F->node[l]) continue;
    long const n = (long)F->t->ext[l][0] * F->t->ext[l][1] * F->t->ext[l][2];
    for (long x = 0; x < n; ++x) free(F->node[l][x]);
    free(F->node[l]);
  }
}

static long lf_cell(int dim, const int y[3]) {
  long c = 0;
  for (int d = 0; d < dim; ++d) c = c * IC + y[d];
  return c;
}

static const double *lf_node(LevelField *F, int L, const int n[3]);

/* value of field e at global cell Y of level L */
static double lf_value(LevelField *F, int L, const int Y0[3], int e) {
  const Geom *g = F->g;
  const Tree *t = F->t;
  int Y[3] = {0, 0, 0}, n[3] = {0, 0, 0}, y[3] = {0, 0, 0};
  for (int d = 0; d < g->dim; ++d) {
    int const top = t->ext[L][d] * IC - 1;
    Y[d] = Y0[d] < 0 ? 0 : (Y0[d] > top ? top : Y0[d]);
    n[d] = Y[d] / IC;
    y[d] = Y[d] - n[d] * IC;
  }
  int const v = t->grid[L][tree_at(t, L, n)];
  if (v >= 0) {
    const double *f = F->src[L] + ((long)v * g->ne + e) * g->cells;
    return f[cidx(g, fic(g, 0) + y[0], fic(g, 1) + y[1], fic(g, 2) + y[2])];
  }
  long const icd = g->dim == 3 ? IC * IC * IC : (g->dim == 2 ? IC * IC : IC);
  return lf_node(F, L, n)[(long)e * icd + lf_cell(g->dim, y)];
}

static const double *lf_node(LevelField *F, int L, const int n[3]) {
  const Geom *g = F->g;
  const Tree *t = F->t;
  int const dim = g->dim;
  long const x = tree_at(t, L, n);
  if (!F->node[L]) {
    long const cnt = (long)t->ext[L][0] * t->ext[L][1] * t->ext[L][2];
    F->node[L] = (double **)calloc((size_t)cnt, sizeof(double *));
  }
  if (F->node[L][x]) return F->node[L][x];
  long const icd = dim == 3 ? IC * IC * IC : (dim == 2 ? IC * IC : IC);
  double *blk = (double *)malloc(sizeof(double) * g->ne * icd);
  int const ext1 = dim > 1 ? IC : 1, ext2 = dim > 2 ? IC : 1;
  if (t->grid[L][x] == -2) {
    /* refined: average of the 2^dim children cells of level L + 1 */
    for (int e = 0; e < g->ne; ++e)
      for (int a = 0; a < IC; ++a)
        for (int b = 0; b < ext1; ++b)
          for (int c = 0; c < ext2; ++c) {
            int const y[3] = {a, b, c};
            double w[8];
            for (int o = 0; o < (1 << dim); ++o) {
              int Y[3] = {0, 0, 0};
              for (int d = 0; d < dim; ++d) Y[d] = 2 * (n[d] * IC + y[d]) + ((o >> d) & 1);
              w[o] = lf_value(F, L + 1, Y, e);
            }
            blk[(long)e * icd + lf_cell(dim, y)] = average_values(dim, w);
          }
  } else {
    /* inside a coarser leaf: predicted from level L - 1 */
    for (int e = 0; e < g->ne; ++e)
      for (int a = 0; a < IC / 2; ++a)
        for (int b = 0; b < (dim > 1 ? IC / 2 : 1); ++b)
          for (int c = 0; c < (dim > 2 ? IC / 2 : 1); ++c) {
            int const q[3] = {a, b, c};
            int P[3] = {0, 0, 0};
            for (int d = 0; d < dim; ++d) P[d] = n[d] * (IC / 2) + q[d];
            double v[125];
            for (int i = -2; i <= 2; ++i)
              for (int j = -2; j <= 2; ++j)
                for (int k = -2; k <= 2; ++k) {
                  int const o[3] = {i, dim > 1 ? j : 0, dim > 2 ? k : 0};
                  int Y[3] = {0, 0, 0};
                  for (int d = 0; d < dim; ++d) Y[d] = P[d] + o[d];
                  PRED_V(i, j, k) = lf_value(F, L - 1, Y, e);
                }
            double out[8];
            predict_children(dim, v, out);
            for (int o = 0; o < (1 << dim); ++o) {
              int y[3] = {0, 0, 0};
              for (int d = 0; d < dim; ++d) y[d] = 2 * q[d] + ((o >> d) & 1);
              blk[(long)e * icd + lf_cell(dim, y)] = out[o];
            }
          }
  }
  F->node[L][x] = blk;
  return blk;
}

/* Face halos (HS layers over the interior extent) of leaf b in pool dst; the
 * neighbours' values come from src[level] (a pool per level). */
static void level_halos(const Geom *g, const Tree *t, int b, double *dst, double *const *src,
                        LevelField *F) {
  int const l = t->level[b], ne = g->ne;
  long const blk = (long)ne * g->cells;
  double *ub = dst + b * blk;
  for (int f = 0; f < 2 * g->dim; ++f) {
    int const d = f / 2, s = (f % 2) ? 1 : -1;
    int p[3];
    for (int e = 0; e < 3; ++e) p[e] = e < g->dim ? t->coord[3 * b + e] : 0;
    p[d] += s;
    int kind, v = -1;
    if (p[d] < 0 || p[d] >= t->ext[l][d]) {
      kind = 0; /* domain face: zero gradient */
    } else {
      v = t->grid[l][tree_at(t, l, p)];
      kind = v >= 0 ? 1 : (v == -2 ? 2 : 3);
    }
    int ext[3];
    for (int e = 0; e < 3; ++e) ext[e] = g->ic[e];
    ext[d] = HS;
    for (int h0 = 0; h0 < ext[0]; ++h0)
      for (int h1 = 0; h1 < ext[1]; ++h1)
        for (int h2 = 0; h2 < ext[2]; ++h2) {
          int hh[3] = {h0, h1, h2};
          /* halo cell in this block, and the neighbour node's interior cell */
          int hc[3], a[3];
          for (int e = 0; e < 3; ++e) {
            hc[e] = fic(g, e) + hh[e];
            a[e] = hh[e];
          }
          hc[d] = s > 0 ? HS + IC + hh[d] : hh[d];
          a[d] = s > 0 ? hh[d] : IC - HS + hh[d];
          long const x = cidx(g, hc[0], hc[1], hc[2]);
          for (int e = 0; e < ne; ++e) {
            double *fo = ub + (long)e * g->cells;
            double val;
            if (kind == 0) {
              int zc[3] = {hc[0], hc[1], hc[2]};
              zc[d] = s > 0 ? HS + IC - 1 : HS;
              val = fo[cidx(g, zc[0], zc[1], zc[2])];
            } else if (kind == 1) {
              const double *fs = src[l] + v * blk + (long)e * g->cells;
              val = fs[cidx(g, fic(g, 0) + a[0], fic(g, 1) + a[1], fic(g, 2) + a[2])];
            } else if (kind == 2) {
              int cc[3], ci[3];
              for (int q = 0; q < 3; ++q) {
                int const o = q < g->dim ? a[q] / (IC / 2) : 0;
                cc[q] = q < g->dim ? 2 * p[q] + o : 0;
                ci[q] = q < g->dim ? fic(g, q) + 2 * (a[q] % (IC / 2)) : 0;
              }
              int const c = t->grid[l + 1][tree_at(t, l + 1, cc)];
              const double *fs = src[l + 1] + c * blk + (long)e * g->cells;
              val = child_average(g, fs, ci[0], ci[1], ci[2]);
            } else {
              int X[3] = {0, 0, 0};
              for (int q = 0; q < g->dim; ++q) X[q] = p[q] * IC + a[q];
              val = lf_value(F, l, X, e);
            }
            fo[x] = val;
          }
        }
  }
}

/* The face halos of every leaf of one snapshot u [nleaf][ne][cells] (interiors
 * read), as a stage of the level step fills them (level_halos with every
 * level's values in u): same-level neighbours copied, finer neighbours
 * averaged, coarser neighbours predicted. Returns tree_build's status. */
int oracle_level_halos(int dim, double *u, int nleaf, const int *level, const int *coord,
                       const int *n0) {
  if (dim < 1 || dim > 3 || nleaf <= 0) return 1;
  Geom g = make_geom(dim);
  Tree tr;
  int const rc = tree_build(&tr, dim, nleaf, level, coord, n0);
  if (rc) {
    tree_free(&tr);
    return rc;
  }
  double *src[MAXLEV];
  for (int l = 0; l < MAXLEV; ++l) src[l] = u;
  LevelField field;
  lf_init(&field, &g, &tr, src);
  /* halos are written, interiors only read: u serves as source and target */
  for (int b = 0; b < nleaf; ++b) level_halos(&g, &tr, b, u, src, &field);
  lf_free(&field);
  tree_free(&tr);
  return 0;
}

/* Face neighbour kind of leaf b across face loc (East 0, West 1, North 2,
 * South 3, Top 4, Bottom 5; boundary_specifications.h:56-63): 0 domain face,
 * 1 same-level leaf, 2 refined node (finer leaves), 3 inside a coarser leaf.
 * p receives the neighbour position at the leaf's level. */
static int face_kind(const Tree *t, int b, int loc, int p[3]) {
  int const l = t->level[b], d = loc / 2, s = (loc % 2) ? -1 : 1;
  for (int e = 0; e < 3; ++e) p[e] = e < t->dim ? t->coord[3 * b + e] : 0;
  p[d] += s;
  if (p[d] < 0 || p[d] >= t->ext[l][d]) return 0;
  int const v = t->grid[l][tree_at(t, l, p)];
  return v >= 0 ? 1 : (v == -2 ? 2 : 3);
}

/* Boundary face fluxes of a leaf, per location and field over the transverse
 * face cells (p1, p2) in increasing dimension order (the jump-buffer layout,
 * space_solver.cpp:155-182), from the flux arrays of block_fluxes. */
static void boundary_fluxes(const Geom *g, double *f[3], double *out) {
  int const ne = g->ne, n2 = IC * IC;
  for (int loc = 0; loc < 2 * g->dim; ++loc) {
    int const d = loc / 2, a = (loc % 2) ? 0 : g->ic[d];
    int const t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
    for (int e = 0; e < ne; ++e)
      for (int p1 = 0; p1 < g->ic[t1]; ++p1)
        for (int p2 = 0; p2 < g->ic[t2]; ++p2) {
          int fi[3];
          fi[d] = a;
          fi[t1] = p1 + 1;
          fi[t2] = p2 + 1;
          out[((long)loc * ne + e) * n2 + p1 * IC + p2] =
              f[d][(long)e * g->faces + fidx(g, fi[0], fi[1], fi[2])];
        }
  }
}

/* number of levels GetLevels(t) returns (modular_algorithm_assembler.cpp:2564-2573) */
static int get_levels_height(unsigned t) { return __builtin_popcount((t + 1) ^ t); }

typedef struct {
  const Geom *g;
  const Eos *e;
  int solver, recon;
  const Tree *t;
  const int *items;
  double *pool;
  double *rhs;
  double *bflux; /* per leaf [6][NE][IC*IC] boundary face fluxes */
  double h0;
} LevelRhsCtx;

static void level_rhs_task(void *vctx, int i, Work *w, double *f[3]) {
  LevelRhsCtx *c = (LevelRhsCtx *)vctx;
  int const b = c->items[i];
  long const blk = (long)c->g->ne * c->g->cells;
  double const h = c->h0 / (double)(1 << c->t->level[b]);
  block_fluxes(c->g, c->e, c->solver, c->recon, c->pool + b * blk, w, f);
  block_divergence(c->g, h, f, c->rhs + b * blk);
  boundary_fluxes(c->g, f, c->bflux + (long)b * 6 * c->g->ne * IC * IC);
}

/* RK3 jump multipliers (runge_kutta_3_TVD.h:42-46) */
static const double rk_jump[3] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
/* TVD-RK2 jump multipliers (runge_kutta_2_TVD.h:40-44) */
static const double rk2_jump[3] = {0.5, 0.5, 0.0};

/* End of micro step tm for the levels >= lu (they just finished a step with
 * a positive level step): AverageJumpBuffer of the finished fine leaves onto
 * their parents' faces, then JumpFluxAdjustment of the finished coarse leaves,
 * then the reset. */
static void level_jump_fluxes(const Geom *g, const Tree *t, double *u, double *jump,
                              double **pjump[MAXLEV], const double *hist, int tm, int lu,
                              double h0) {
  int const ne = g->ne, n2 = IC * IC, dim = g->dim;
  long const jsz = 6L * ne * n2, fsz = (long)ne * n2;
  long const blk = (long)ne * g->cells;
  int done[MAXLEV];
  for (int l = 0; l <= t->lmax; ++l) {
    double dtl = 0.0;
    if (l >= lu)
      for (int k = tm; k > tm - (1 << (t->lmax - l)); --k) dtl += hist[k];
    done[l] = dtl > 0.0;
  }
  /* averaging down (multiresolution.cpp:47-128), finished fine leaves */
  for (int b = 0; b < t->nleaf; ++b) {
    int const l = t->level[b];
    if (l == 0 || !done[l]) continue;
    for (int loc = 0; loc < 2 * dim; ++loc) {
      int pn[3];
      if (face_kind(t, b, loc, pn) != 3) continue;
      int pc[3] = {0, 0, 0}, oc[3] = {0, 0, 0};
      for (int e = 0; e < dim; ++e) {
        pc[e] = t->coord[3 * b + e] >> 1;
        oc[e] = t->coord[3 * b + e] & 1;
      }
      long const pidx = tree_at(t, l - 1, pc);
      double **slot = &pjump[l - 1][pidx];
      if (!*slot) *slot = (double *)calloc((size_t)jsz, sizeof(double));
      double *pj = *slot + (long)loc * fsz;
      double *cj = jump + (long)b * jsz + (long)loc * fsz;
      int const d = loc / 2, t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
      int const n1 = g->ic[t1] > 1 ? IC / 2 : 1, n2c = g->ic[t2] > 1 ? IC / 2 : 1;
      int const o1 = t1 < dim ? oc[t1] * (IC / 2) : 0, o2 = t2 < dim ? oc[t2] * (IC / 2) : 0;
      for (int e = 0; e < ne; ++e)
        for (int i = 0; i < n1; ++i)
          for (int j = 0; j < n2c; ++j) {
            const double *c = cj + (long)e * n2;
            double v;
            if (dim == 1)
              v = c[0];
            else if (dim == 2)
              v = (c[(2 * i) * IC] + c[(2 * i + 1) * IC]) * 0.5;
            else
              v = ((c[(2 * i) * IC + 2 * j] + c[(2 * i + 1) * IC + 2 * j + 1]) +
                   (c[(2 * i + 1) * IC + 2 * j] + c[(2 * i) * IC + 2 * j + 1])) * 0.25;
            pj[(long)e * n2 + (o1 + i) * IC + (o2 + j)] += v;
          }
      for (long x = 0; x < fsz; ++x) cj[x] = 0.0;
    }
  }
  /* exchange and correction (modular_algorithm_assembler.cpp:1410-1636) */
  for (int b = 0; b < t->nleaf; ++b) {
    int const l = t->level[b];
    if (!done[l]) continue;
    int kinds[6] = {0, 0, 0, 0, 0, 0}, any = 0;
    double *pj[6] = {0, 0, 0, 0, 0, 0};
    for (int loc = 0; loc < 2 * dim; ++loc) {
      int pn[3];
      kinds[loc] = face_kind(t, b, loc, pn);
      if (kinds[loc] != 2) continue;
      any = 1;
      double **slot = &pjump[l][tree_at(t, l, pn)];
      if (!*slot) *slot = (double *)calloc((size_t)jsz, sizeof(double));
      pj[loc] = *slot + (long)(loc ^ 1) * fsz; /* the neighbour's opposite face */
    }
    if (!any) continue;
    double const ocs = 1.0 / (h0 / (double)(1 << l));
    double *ub = u + b * blk;
    for (int e = 0; e < ne; ++e)
      for (int i = 0; i < g->ic[0]; ++i)
        for (int j = 0; j < g->ic[1]; ++j)
          for (int k = 0; k < g->ic[2]; ++k) {
            int const a[3] = {i, j, k};
            double cf[6] = {0, 0, 0, 0, 0, 0}, ff[6] = {0, 0, 0, 0, 0, 0};
            int touched = 0;
            for (int loc = 0; loc < 2 * dim; ++loc) {
              if (kinds[loc] != 2) continue;
              int const d = loc / 2, high = (loc % 2) == 0;
              if (a[d] != (high ? IC - 1 : 0)) continue;
              int const t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
              long const x = (long)e * n2 + a[t1] * IC + (t2 < 3 ? a[t2] : 0);
              double const dir = high ? -1.0 : 1.0;
              cf[loc] = jump[(long)b * jsz + (long)loc * fsz + x] * ocs * dir;
              ff[loc] = pj[loc][x] * ocs * dir;
              touched = 1;
            }
            if (!touched) continue;
            double *cell = ub + (long)e * g->cells + cidx(g, i + fic(g, 0), j + fic(g, 1), k + fic(g, 2));
            *cell -= cms3(cf[0] + cf[1], cf[2] + cf[3], cf[4] + cf[5]);
            *cell += cms3(ff[0] + ff[1], ff[2] + ff[3], ff[4] + ff[5]);
          }
    for (int loc = 0; loc < 2 * dim; ++loc) {
      if (kinds[loc] != 2) continue;
      double *cj = jump + (long)b * jsz + (long)loc * fsz;
      for (long x = 0; x < fsz; ++x) {
        cj[x] = 0.0;
        pj[loc][x] = 0.0;
      }
    }
  }
}

int oracle_levels_run(int dim, int solver, int recon, double *u, int nleaf, const int *level,
                      const int *coord, const int *n0, double h0, double gamma, double B,
                      int safe, double cfl, double t_end, int max_macro, int nthreads,
                      double *t_io, int *macro_done, double *dt_log) {
  if (dim < 1 || dim > 3 || nleaf <= 0) return 1;
  Geom g = make_geom(dim);
  Eos e = {dim, gamma, B, safe};
  Tree tr;
  int rc = tree_build(&tr, dim, nleaf, level, coord, n0);
  if (rc) {
    tree_free(&tr);
    return rc;
  }
  int const lmax = tr.lmax, nmicro = 1 << lmax;
  long const blk = (long)g.ne * g.cells, n = (long)nleaf * blk;
  double *pb = (double *)malloc(sizeof(double) * n);
  double *pc = (double *)malloc(sizeof(double) * n);
  double *rhs = (double *)calloc((size_t)n, sizeof(double));
  int *items = (int *)malloc(sizeof(int) * nleaf);
  double *hist = (double *)malloc(sizeof(double) * nmicro);
  long const jsz = 6L * g.ne * IC * IC; /* one leaf's six jump buffers */
  double *bflux = (double *)calloc((size_t)nleaf * jsz, sizeof(double));
  double *jump = (double *)calloc((size_t)nleaf * jsz, sizeof(double));
  /* jump buffers of refined nodes (the parents' faces), per level and node */
  double **pjump[MAXLEV] = {0};
  int ok = pb && pc && rhs && items && hist && bflux && jump;
  for (int l = 0; ok && l <= tr.lmax; ++l) {
    pjump[l] = (double **)calloc((size_t)tr.ext[l][0] * tr.ext[l][1] * tr.ext[l][2], sizeof(double *));
    ok = pjump[l] != NULL;
  }
  if (!ok) {
    free(pb); free(pc); free(rhs); free(items); free(hist); free(bflux); free(jump);
    for (int l = 0; l < MAXLEV; ++l) free(pjump[l]);
    tree_free(&tr);
    return 3;
  }
  memcpy(pb, u, sizeof(double) * n);
  memcpy(pc, u, sizeof(double) * n);
  double *pool_in[3] = {u, pb, pc};
  double *pool_out[3] = {pb, pc, u};
  /* SSP-RK3 or TVD-RK2 (the last stage writes the state pool) */
  int const nst = rk_stages();
  const double(*rka)[2] = g_integrator == TI_RK2 ? rk2_a : rk3_a;
  const double *const rkc = g_integrator == TI_RK2 ? rk2_c : rk3_c;
  const double *const rkj = g_integrator == TI_RK2 ? rk2_jump : rk_jump;
  if (nst == 2) pool_out[1] = u;
  double const h_fine = h0 / (double)nmicro;
  double t = *t_io;
  int macro = 0, logged = 0;
  while (t < t_end && (max_macro <= 0 || macro < max_macro)) {
    for (int tm = 0; tm < nmicro; ++tm) {
      double cur = t;
      for (int k = 0; k < tm; ++k) cur = cur + hist[k];
      double dt;
      oracle_timestep(dim, u, nleaf, gamma, B, safe, h_fine, cfl, cur, t_end, &dt);
      hist[tm] = dt;
      if (dt_log) dt_log[logged] = dt;
      ++logged;
      int const lu = lmax - get_levels_height((unsigned)tm) + 1;
      int const lf0 = tm == 0 ? 0 : lmax - get_levels_height((unsigned)(tm - 1)) + 1;
      for (int s = 0; s < nst; ++s) {
        int const lflux = s == 0 ? lf0 : lu;
        double *src[MAXLEV];
        for (int l = 0; l <= lmax; ++l) src[l] = (s > 0 && l >= lu) ? pool_in[s] : u;
        int ni = 0;
        LevelField field;
        lf_init(&field, &g, &tr, src);
        for (int b = 0; b < nleaf; ++b)
          if (level[b] >= lflux) {
            level_halos(&g, &tr, b, pool_in[s], src, &field);
            items[ni++] = b;
          }
        lf_free(&field);
        if (glf_selected(solver)) glf_maxima_leaves(&g, &e, src, level, items, ni);
        LevelRhsCtx c = {&g, &e, solver, recon, &tr, items, pool_in[s], rhs, bflux, h0};
        parallel_blocks(&g, ni, nthreads, level_rhs_task, &c);
        for (int b = 0; b < nleaf; ++b) {
          int const l = level[b];
          if (l < lu) continue;
          double dtl = 0.0;
          for (int k = tm; k > tm - (1 << (lmax - l)); --k) dtl += hist[k];
          if (!(dtl > 0.0)) continue;
          double const step = rkc[s] * (0.0 + dtl);
          double const m0 = rka[s][0], m1 = rka[s][1];
          const double *ui = pool_in[s] + b * blk, *u0 = u + b * blk, *r = rhs + b * blk;
          double *uo = pool_out[s] + b * blk;
          for (int f = 0; f < g.ne; ++f)
            for (int i = fic(&g, 0); i <= lic(&g, 0); ++i)
              for (int j = fic(&g, 1); j <= lic(&g, 1); ++j)
                for (int k = fic(&g, 2); k <= lic(&g, 2); ++k) {
                  long const x = (long)f * g.cells + cidx(&g, i, j, k);
                  double v = ui[x];
                  if (s != 0) v = m0 * v + m1 * u0[x];
                  uo[x] = v + step * r[x];
                }
          /* IntegrateJumpConservatives: jump faces integrate their fluxes */
          double const jstep = rkj[s] * dtl;
          for (int loc = 0; loc < 2 * dim; ++loc) {
            int pn[3];
            int const kind = face_kind(&tr, b, loc, pn);
            if (kind < 2) continue;
            double *jb = jump + (long)b * jsz + (long)loc * g.ne * IC * IC;
            const double *fb = bflux + (long)b * jsz + (long)loc * g.ne * IC * IC;
            for (long x = 0; x < (long)g.ne * IC * IC; ++x) jb[x] += jstep * fb[x];
          }
        }
      }
      level_jump_fluxes(&g, &tr, u, jump, pjump, hist, tm, lu, h0);
    }
    double sum = 0.0;
    for (int k = 0; k < nmicro; ++k) sum = sum + hist[k];
    t = t + sum;
    ++macro;
  }
  free(pb); free(pc); free(rhs); free(items); free(hist); free(bflux); free(jump);
  for (int l = 0; l < MAXLEV; ++l) {
    if (pjump[l])
      for (long x = 0; x < (long)tr.ext[l][0] * tr.ext[l][1] * tr.ext[l][2]; ++x) free(pjump[l][x]);
    free(pjump[l]);
  }
  tree_free(&tr);
  *t_io = t;
  *macro_done = macro;
  return 0;
}

/* Selects stencil, Riemann solver, signal speed and flux splitting (values of
 * the reference's enums); 1 for an unknown value. */
int oracle_set_options(int stencil, int riemann, int signal, int splitting) {
  if (stencil != ST_WENO5 && stencil != ST_WENO5Z && stencil != ST_TENO5 && stencil != ST_WENO7 &&
      stencil != ST_WENO3 && stencil != ST_FIRST_ORDER)
    return 1;
  if (riemann < RS_HLLC || riemann > RS_HLL) return 1;
  if (signal < SS_EINFELDT || signal > SS_ARITHMETIC) return 1;
  if (splitting != FSP_ROE && splitting != FSP_LLF && splitting != FSP_GLF &&
      splitting != FSP_ROE_M && splitting != FSP_LLF_M)
    return 1;
  g_stencil = stencil;
  g_riemann = riemann;
  g_signal = signal;
  g_splitting = splitting;
  return 0;
}
