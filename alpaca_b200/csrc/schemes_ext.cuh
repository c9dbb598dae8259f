// Further instantiations of the reference's plugin surface, selected at run
// time in FP64 beside the compiled default (WENO5 + HLLC + Einfeldt, Roe
// splitting):
//   reconstruction stencils  WENO5-Z, TENO5, WENO3, first order
//                            (stencils/spatial_reconstruction_stencils/)
//   Riemann solvers          HLL, HLLC-LM (solvers/convective_term_contributions/
//                            riemann_solvers/hll_riemann_solver.h,
//                            hllc_lm_riemann_solver.h)
//   signal speeds            Davis, Toro, arithmetic (hll_signal_speed_calculator.h)
//   flux splitting           Roe-M, local Lax-Friedrichs, LLF-M
//                            (solvers/eigendecomposition.h:416-454)
// Every expression keeps the reference's operation order, so the strict build
// reproduces the reference bit for bit except where the reference calls
// std::pow (Toro) or std::sin (HLLC-LM), whose CUDA versions may round
// differently in the last bit.
#pragma once

#include "kernels.cuh"
#include "numerics.cuh"

namespace alp {

// WENO5-Z (weno5_z.h:88-150): tau = |beta1 - beta3|, alpha_k = d_k (1 + tau /
// (beta_k + eps)), eps = machine epsilon.
__device__ __forceinline__ double weno5z_core(double v1, double v2, double v3, double v4,
                                              double v5) {
  double const c1 = 13.0 / 12.0, c2 = 0.25;
  double const s11 = v1 + -2.0 * v2 + v3;
  double const s12 = v1 + -4.0 * v2 + 3.0 * v3;
  double const s1 = c1 * s11 * s11 + c2 * s12 * s12;
  double const s21 = v2 + -2.0 * v3 + v4;
  double const s22 = v2 + -1.0 * v4;
  double const s2 = c1 * s21 * s21 + c2 * s22 * s22;
  double const s31 = v3 + -2.0 * v4 + v5;
  double const s32 = 3.0 * v3 + -4.0 * v4 + v5;
  double const s3 = c1 * s31 * s31 + c2 * s32 * s32;
  double const tau = fabs(s1 - s3);
  double const a1 = 0.1 * (1.0 + quot(tau, s1 + DBL_EPSILON));
  double const a2 = 0.6 * (1.0 + quot(tau, s2 + DBL_EPSILON));
  double const a3 = 0.3 * (1.0 + quot(tau, s3 + DBL_EPSILON));
  double const one_a_sum = quot(1.0, a1 + a2 + a3);
  double const w1 = a1 * one_a_sum, w2 = a2 * one_a_sum, w3 = a3 * one_a_sum;
  return w1 * (2.0 / 6.0 * v1 + -7.0 / 6.0 * v2 + 11.0 / 6.0 * v3) +
         w2 * (-1.0 / 6.0 * v2 + 5.0 / 6.0 * v3 + 2.0 / 6.0 * v4) +
         w3 * (2.0 / 6.0 * v3 + 5.0 / 6.0 * v4 + -1.0 / 6.0 * v5);
}

// TENO5 (teno5.h:98-180): smoothness of the candidate stencils, alpha_k =
// (1 + tau5 / (beta_k + eps))^6, cut-off C_T = 1e-5 on the normalised alpha,
// then the ideal weights (0.6, 0.3, 0.1) of the surviving stencils.
__device__ __forceinline__ double teno5_core(double v1, double v2, double v3, double v4,
                                             double v5) {
  double const c1 = 13.0 / 12.0, c2 = 0.25;
  double const s11 = v2 + -2.0 * v3 + v4;
  double const s12 = v2 + -1.0 * v4;
  double const s1 = c1 * s11 * s11 + c2 * s12 * s12;
  double const s21 = v3 + -2.0 * v4 + v5;
  double const s22 = 3.0 * v3 + -4.0 * v4 + v5;
  double const s2 = c1 * s21 * s21 + c2 * s22 * s22;
  double const s31 = v1 + -2.0 * v2 + v3;
  double const s32 = v1 + -4.0 * v2 + 3.0 * v3;
  double const s3 = c1 * s31 * s31 + c2 * s32 * s32;
  double const tau5 = fabs(s3 - s2);
  double a1 = 1.0 + quot(tau5, s1 + DBL_EPSILON);
  double a2 = 1.0 + quot(tau5, s2 + DBL_EPSILON);
  double a3 = 1.0 + quot(tau5, s3 + DBL_EPSILON);
  a1 *= (a1 * a1);
  a2 *= (a2 * a2);
  a3 *= (a3 * a3);
  a1 *= a1;
  a2 *= a2;
  a3 *= a3;
  double const one_a_sum = quot(1.0, a1 + a2 + a3);
  double const b1 = a1 * one_a_sum < 1.0e-5 ? 0.0 : 1.0;
  double const b2 = a2 * one_a_sum < 1.0e-5 ? 0.0 : 1.0;
  double const b3 = a3 * one_a_sum < 1.0e-5 ? 0.0 : 1.0;
  double const var1 = -1.0 * v2 + 5.0 * v3 + 2.0 * v4;
  double const var2 = 2.0 * v3 + 5.0 * v4 + -1.0 * v5;
  double const var3 = 2.0 * v1 + -7.0 * v2 + 11.0 * v3;
  double const w1 = 0.6 * b1, w2 = 0.3 * b2, w3 = 0.1 * b3;
  double const one_w_sum = quot(1.0, w1 + w2 + w3);
  return ((w1 * one_w_sum) * var1 + (w2 * one_w_sum) * var2 + (w3 * one_w_sum) * var3) *
         (1.0 / 6.0);
}

// WENO3 (weno3.h:66-100) on three cells, eps = machine epsilon.
__device__ __forceinline__ double weno3_core(double v1, double v2, double v3) {
  double const s11 = -1.0 * v1 + v2;
  double const s1 = s11 * s11;
  double const s21 = -1.0 * v2 + v3;
  double const s2 = s21 * s21;
  double const a1 = quot(1.0 / 3.0, (s1 + DBL_EPSILON) * (s1 + DBL_EPSILON));
  double const a2 = quot(2.0 / 3.0, (s2 + DBL_EPSILON) * (s2 + DBL_EPSILON));
  double const one_a_sum = quot(1.0, a1 + a2);
  double const w1 = a1 * one_a_sum, w2 = a2 * one_a_sum;
  return w1 * (-1.0 / 2.0 * v1 + 3.0 / 2.0 * v2) + w2 * (1.0 / 2.0 * v2 + 1.0 / 2.0 * v3);
}

// Reconstruction of the 6-cell array a (cells i-2..i+3 around face i+1/2) with
// UpwindLeft (right = false) or UpwindRight evaluation properties
// (stencils/apply_wrapper.h:47-57); narrower stencils use the middle cells.
// WENO7-JS (weno7.h:21-212; coefficients of Balsara & Shu 2000): v1..v7 the
// cells i-3..i+3 seen from the upwind side, eps 1e-10, the reference's
// association order.
__device__ __forceinline__ double weno7_core(double v1, double v2, double v3, double v4,
                                             double v5, double v6, double v7) {
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
  double const a1 = quot(1.0 / 35.0, (s1 + eps) * (s1 + eps));
  double const a2 = quot(12.0 / 35.0, (s2 + eps) * (s2 + eps));
  double const a3 = quot(18.0 / 35.0, (s3 + eps) * (s3 + eps));
  double const a4 = quot(4.0 / 35.0, (s4 + eps) * (s4 + eps));
  double const one_a_sum = quot(1.0, a1 + a2 + a3 + a4);
  double const w1 = a1 * one_a_sum, w2 = a2 * one_a_sum, w3 = a3 * one_a_sum,
               w4 = a4 * one_a_sum;
  return w1 * (-3.0 / 12.0 * v1 + 13.0 / 12.0 * v2 + -23.0 / 12.0 * v3 + 25.0 / 12.0 * v4) +
         w2 * (1.0 / 12.0 * v2 + -5.0 / 12.0 * v3 + 13.0 / 12.0 * v4 + 3.0 / 12.0 * v5) +
         w3 * (-1.0 / 12.0 * v3 + 7.0 / 12.0 * v4 + 7.0 / 12.0 * v5 + -1.0 / 12.0 * v6) +
         w4 * (3.0 / 12.0 * v4 + 13.0 / 12.0 * v5 + -5.0 / 12.0 * v6 + 1.0 / 12.0 * v7);
}

// a: the N cells of the stencil line with the face's left cell i at N/2 - 1
// (N = 6: i-2..i+3, N = 8: i-3..i+4); the five- and three-point stencils read
// the middle cells.
template <int N>
__device__ __forceinline__ double reconstruct(int stencil, double const (&a)[N], bool right) {
  constexpr int o = N / 2 - 3;  // a[o + k]: cell i - 2 + k
  switch (stencil) {
    case ST_WENO7:
      if constexpr (N >= 8)
        return right ? weno7_core(a[o + 6], a[o + 5], a[o + 4], a[o + 3], a[o + 2], a[o + 1], a[o])
                     : weno7_core(a[o - 1], a[o], a[o + 1], a[o + 2], a[o + 3], a[o + 4], a[o + 5]);
      else
        return 0.0;  // not reachable: WENO7 runs with 8-cell stencils
    case ST_WENO5Z:
      return right ? weno5z_core(a[o + 5], a[o + 4], a[o + 3], a[o + 2], a[o + 1])
                   : weno5z_core(a[o], a[o + 1], a[o + 2], a[o + 3], a[o + 4]);
    case ST_TENO5:
      return right ? teno5_core(a[o + 5], a[o + 4], a[o + 3], a[o + 2], a[o + 1])
                   : teno5_core(a[o], a[o + 1], a[o + 2], a[o + 3], a[o + 4]);
    case ST_WENO3:
      return right ? weno3_core(a[o + 4], a[o + 3], a[o + 2])
                   : weno3_core(a[o + 1], a[o + 2], a[o + 3]);
    case ST_FIRST_ORDER:
      return right ? a[o + 3] : a[o + 2];
    default:
      return right ? weno5_core(a[o + 5], a[o + 4], a[o + 3], a[o + 2], a[o + 1])
                   : weno5_core(a[o], a[o + 1], a[o + 2], a[o + 3], a[o + 4]);
  }
}

// CalculateSignalSpeed (hll_signal_speed_calculator.h:40-140): unclamped left
// and right wave speeds.
__device__ __forceinline__ void signal_speeds(int which, double rl, double rr, double ul,
                                              double ur, double pl, double pr, double cl,
                                              double cr, double gamma, double &sl,
                                              double &sr) {
  if (which == SS_ARITHMETIC) {
    double const cf = 0.5 * (cl + cr);
    double const uf = 0.5 * (ul + ur);
    sl = dmin(uf - cf, ul - cl);
    sr = dmax(uf + cf, ur + cr);
  } else if (which == SS_DAVIS) {
    sl = dmin(ul - cl, ur - cr);
    sr = dmax(ul + cl, ur + cr);
  } else if (which == SS_TORO) {
    double const z = quot(gamma - 1.0, 2.0 * gamma);
    double const p_star =
        pow(quot((cl + cr) - 0.5 * (ur - ul) * (gamma - 1.0),
                 quot(cl, pow(pl, z)) + quot(cr, pow(pr, z))),
            quot(1.0, z));
    double ql = 1.0, qr = 1.0;
    if (p_star > pl) ql = sqrt(1.0 + quot(gamma + 1.0, 2.0 * gamma) * (quot(p_star, pl) - 1.0));
    if (p_star > pr) qr = sqrt(1.0 + quot(gamma + 1.0, 2.0 * gamma) * (quot(p_star, pr) - 1.0));
    sl = ul - cl * ql;
    sr = ur + cr * qr;
  } else {  // Einfeldt
    double const srl = sqrt(rl), srr = sqrt(rr);
    double const rho_div = quot(1.0, srl + srr);
    double const u_roe = ((ul * srl) + (ur * srr)) * rho_div;
    double const c_e = sqrt(((cl * cl * srl) + (cr * cr * srr)) * rho_div +
                            (0.5 * srl * srr * rho_div * rho_div) * (ur - ul) * (ur - ul));
    sl = dmin(u_roe - c_e, ul - cl);
    sr = dmax(u_roe + c_e, ur + cr);
  }
}

// HLLC, HLLC-LM and HLL with any signal speed. Reconstructed conservatives
// cl / cr, their pressures and principal velocities and 1/density.
template <int DIM, int DIR>
__device__ __forceinline__ void riemann_ext(int solver, int speeds, Eos const &e,
                                            double const (&cl)[DIM + 2],
                                            double const (&cr)[DIM + 2], double pres_l,
                                            double pres_r, double vel_l, double vel_r,
                                            double one_rl, double one_rr,
                                            double (&flux)[DIM + 2]) {
  constexpr int NE = DIM + 2;
  constexpr int mP = MOMX + DIR;
  double const c_l = eos_speed_of_sound<double>(e, cl[MASS], pres_l, one_rl);
  double const c_r = eos_speed_of_sound<double>(e, cr[MASS], pres_r, one_rr);
  double sls, srs;
  signal_speeds(speeds, cl[MASS], cr[MASS], vel_l, vel_r, pres_l, pres_r, c_l, c_r, e.gamma, sls,
                srs);
  double fl[NE], fr[NE];
  fl[MASS] = cl[mP];
  fr[MASS] = cr[mP];
  fl[mP] = ((cl[mP] * cl[mP]) * one_rl) + pres_l;
  fr[mP] = ((cr[mP] * cr[mP]) * one_rr) + pres_r;
  fl[ENERGY] = vel_l * (cl[ENERGY] + pres_l);
  fr[ENERGY] = vel_r * (cr[ENERGY] + pres_r);
#pragma unroll
  for (int d = 0; d < DIM - 1; ++d) {
    int const mm = MOMX + (d == 0 ? Minor<DIR>::m1 : Minor<DIR>::m2);
    fl[mm] = vel_l * cl[mm];
    fr[mm] = vel_r * cr[mm];
  }
  if (solver == RS_HLL) {
    // hll_riemann_solver.h:96-150
    double const sl = dmin(sls, 0.0), sr = dmax(srs, 0.0);
#pragma unroll
    for (int n = 0; n < NE; ++n)
      flux[n] = quot(((sr * fl[n]) - (sl * fr[n])) + ((sr * sl) * (cr[n] - cl[n])), sr - sl);
    return;
  }
  bool const lm = solver == RS_HLLC_LM;
  // HLLC clamps the speeds after the contact speed and star states; HLLC-LM
  // uses the unclamped speeds throughout (hllc_lm_riemann_solver.h:96-114)
  double const s_star = quot((pres_r - pres_l) + (cl[mP] * (sls - vel_l) - cr[mP] * (srs - vel_r)),
                             cl[MASS] * (sls - vel_l) - cr[MASS] * (srs - vel_r));
  double const sl = lm ? sls : dmin(sls, 0.0);
  double const sr = lm ? srs : dmax(srs, 0.0);
  double const chi_l = quot(sls - vel_l, sls - s_star);
  double const chi_r = quot(srs - vel_r, srs - s_star);
  double ql[NE], qr[NE];
  ql[MASS] = cl[MASS] * chi_l;
  qr[MASS] = cr[MASS] * chi_r;
  ql[mP] = cl[MASS] * chi_l * s_star;
  qr[mP] = cr[MASS] * chi_r * s_star;
  ql[ENERGY] = cl[MASS] * chi_l *
               (cl[ENERGY] * one_rl + (s_star - vel_l) * (s_star + quot(pres_l, cl[MASS] * (sl - vel_l))));
  qr[ENERGY] = cr[MASS] * chi_r *
               (cr[ENERGY] * one_rr + (s_star - vel_r) * (s_star + quot(pres_r, cr[MASS] * (sr - vel_r))));
#pragma unroll
  for (int d = 0; d < DIM - 1; ++d) {
    int const mm = MOMX + (d == 0 ? Minor<DIR>::m1 : Minor<DIR>::m2);
    ql[mm] = chi_l * cl[mm];
    qr[mm] = chi_r * cr[mm];
  }
  if (!lm) {
    double const sg = double((0.0 < s_star) - (s_star < 0.0));
#pragma unroll
    for (int n = 0; n < NE; ++n) {
      double const fsl = fl[n] + (sl * (ql[n] - cl[n]));
      double const fsr = fr[n] + (sr * (qr[n] - cr[n]));
      flux[n] = (0.5 * (1.0 + sg) * fsl + 0.5 * (1.0 - sg) * fsr);
    }
    return;
  }
  // low-Mach activation (hllc_lm_riemann_solver.h:180-198), Ma limit 0.1
  double const ma = dmin(0.1, dmax(fabs(quot(vel_l, c_l)), fabs(quot(vel_r, c_r))));
  double const act = sin((ma / 0.1) * 1.57079632679489661923);
#pragma unroll
  for (int n = 0; n < NE; ++n) {
    if (sl >= 0.0) {
      flux[n] = fl[n];
    } else if (sr <= 0.0) {
      flux[n] = fr[n];
    } else {
      flux[n] = 0.5 * ((fl[n] + fr[n]) - (((act * sr) * (cr[n] - qr[n]) + (act * sl) * (cl[n] - ql[n])) +
                                          fabs(s_star) * (qr[n] - ql[n])));
    }
  }
}

// Scheme policies of face_compute. The default one is the compiled hot path;
// ExtPolicy dispatches on SchemeOptions at run time (FP64 only).
struct DefaultPolicy {
  template <typename T> __device__ __forceinline__ T left(T const (&a)[6]) const {
    return weno5_left(a);
  }
  template <typename T> __device__ __forceinline__ T right(T const (&a)[6]) const {
    return weno5_right(a);
  }
  template <typename T>
  __device__ __forceinline__ void pair(T const (&a)[6], T &l, T &r) const {
    weno5_pair(a, l, r);
  }
  template <typename T>
  __device__ __forceinline__ void two(T const (&a)[6], T const (&b)[6], T &l, T &r) const {
    weno5_two(a, b, l, r);
  }
  template <int DIM, int DIR, typename T>
  __device__ __forceinline__ void riemann(Eos const &e, T const (&cl)[DIM + 2],
                                          T const (&cr)[DIM + 2], T pl, T pr, T vl, T vr,
                                          T one_l, T one_r, T (&flux)[DIM + 2]) const {
    hllc<DIM, DIR, T>(e, cl, cr, pl, pr, vl, vr, one_l, one_r, flux);
  }
  // flux-splitting eigenvalues |u - c|, |u|, |u + c| of the Roe average
  template <int DIM, int DIR, typename T>
  __device__ __forceinline__ void fs_eigenvalues(Eos const &, Roe<T> const &r,
                                                 CellPrims<DIM, DIR> const &,
                                                 CellPrims<DIM, DIR> const &, T &e0, T &elin,
                                                 T &e1) const {
    e0 = fabs(r.up - r.c);
    e1 = fabs(r.up + r.c);
    elin = fabs(r.up);
  }
};

struct ExtPolicy {
  SchemeOptions o;
  double glf[3] = {0.0, 0.0, 0.0};  // GlobalLaxFriedrichs wave speeds of the block's case
  template <int N> __device__ __forceinline__ double left(double const (&a)[N]) const {
    return reconstruct(o.stencil, a, false);
  }
  template <int N> __device__ __forceinline__ double right(double const (&a)[N]) const {
    return reconstruct(o.stencil, a, true);
  }
  template <int N>
  __device__ __forceinline__ void pair(double const (&a)[N], double &l, double &r) const {
    l = left(a);
    r = right(a);
  }
  template <int N>
  __device__ __forceinline__ void two(double const (&a)[N], double const (&b)[N], double &l,
                                      double &r) const {
    l = left(a);
    r = right(b);
  }
  template <int DIM, int DIR, typename T>
  __device__ __forceinline__ void riemann(Eos const &e, double const (&cl)[DIM + 2],
                                          double const (&cr)[DIM + 2], double pl, double pr,
                                          double vl, double vr, double one_l, double one_r,
                                          double (&flux)[DIM + 2]) const {
    riemann_ext<DIM, DIR>(o.riemann, o.signal, e, cl, cr, pl, pr, vl, vr, one_l, one_r, flux);
  }
  // eigendecomposition.h:416-454
  template <int DIM, int DIR, typename T>
  __device__ __forceinline__ void fs_eigenvalues(Eos const &e, Roe<double> const &r,
                                                 CellPrims<DIM, DIR> const &pt,
                                                 CellPrims<DIM, DIR> const &pn, double &e0,
                                                 double &elin, double &e1) const {
    double const phi = 5.0;  // FluxSplittingSettings::low_mach_number_limit_factor
    if (o.splitting == FSP_ROE_M) {
      double const cm = dmin(r.c, phi * fabs(r.up));
      e0 = fabs(r.up - cm);
      elin = fabs(r.up);
      e1 = fabs(r.up + cm);
    } else if (o.splitting == FSP_LLF || o.splitting == FSP_LLF_M) {
      double ct = eos_speed_of_sound<double>(e, pt.rho, pt.p, pt.one_rho);
      double cn = eos_speed_of_sound<double>(e, pn.rho, pn.p, pn.one_rho);
      if (o.splitting == FSP_LLF_M) {
        ct = dmin(phi * fabs(pt.up), ct);
        cn = dmin(phi * fabs(pn.up), cn);
      }
      e0 = dmax(fabs(pt.up - ct), fabs(pn.up - cn));
      elin = dmax(fabs(pt.up), fabs(pn.up));
      e1 = dmax(fabs(pt.up + ct), fabs(pn.up + cn));
    } else if (o.splitting == FSP_GLF) {
      // the x maxima in every direction (eigendecomposition.h:457-460)
      e0 = glf[0];
      elin = glf[1];
      e1 = glf[2];
    } else {
      e0 = fabs(r.up - r.c);
      e1 = fabs(r.up + r.c);
      elin = fabs(r.up);
    }
  }
};

}  // namespace alp
