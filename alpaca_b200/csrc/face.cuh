// Per-face flux of the block right-hand side, shared by the face-flux kernels
// (kernels.cu) and the fused tile-stage kernel (tile_step.cu): both evaluate
// every face through face_compute, so they produce the same bits.
#pragma once

#include <cfloat>

#include "kernels.cuh"

// The FP32-flux branches return early, which leaves the shared FP64 tail
// unreachable in those instantiations.
#pragma nv_diag_suppress 128
#include "numerics.cuh"
#include "schemes_ext.cuh"

namespace alp {

// Structural nonzeros of the left eigenvector matrix row n, column l
// (eigendecomposition.h:316-359).
template <int DIM, int DIR>
__host__ __device__ constexpr bool left_nonzero(int n, int l) {
  // the rows of the two acoustic waves and of the principal-momentum wave are full
  if (n == 0 || n == DIM + 1 || n == DIM) return true;
  // minor-momentum waves: mass and their own momentum only
  return l == MASS || l == MOMX + (n == 1 ? Minor<DIR>::m1 : Minor<DIR>::m2);
}


// Flux of one face from its 6-cell stencil (the reference's per-face work:
// FiniteVolumeScheme::ComputeFluxes<DIR> with the selected reconstruction and
// HLLC, or FluxSplittingScheme::ComputeFluxes<DIR>). Writes the flux in double
// to fd and returns false for a face the reference skips (invalid
// reconstructed state, finite_volume_scheme.cpp:218-225) or whose Roe average
// has a non-positive density (eigendecomposition.h:244).
// P selects reconstruction stencil, Riemann solver and splitting eigenvalues
// (DefaultPolicy: WENO5, HLLC/Einfeldt, Roe; ExtPolicy: run-time choice, FP64).
template <int DIM, int DIR, int SCHEME, typename T, typename P = DefaultPolicy, int W = 6>
__device__ __forceinline__ bool face_compute(Eos const &eos, double B,
                                             double const (&cons)[W][DIM + 2],
                                             double (&fd)[DIM + 2], P const &pol = P()) {
  constexpr int NE = DIM + 2;
  T flux[NE];
  bool valid = true;
  constexpr int mP = MOMX + DIR;
  constexpr int C = W / 2 - 1;  // the face's left cell i in the stencil

  if constexpr (SCHEME == FV_CHAR || SCHEME == FS_ROE) {
    auto const pt = cell_prims<DIM, DIR>(eos, cons[C]);
    auto const pn = cell_prims<DIM, DIR>(eos, cons[C + 1]);
    if (!(pt.rho > 0.0) || !(pn.rho > 0.0)) valid = false;
    Roe<T> const r = roe_average<DIM, DIR, T>(eos, pt, pn);
    T ch[2][NE];
    if constexpr (SCHEME == FV_CHAR && sizeof(T) == 4) {
      // FP32 form: characteristic projection and WENO5 of the increments
      // U_m - U_i against the face's left cell i (WENO5 is translation
      // invariant and R L = I), the left cell's state added back in double.
      // The increments are formed in double and converted once each, for all
      // five characteristic fields.
      float du[W][NE];
#pragma unroll
      for (int m = 0; m < W; ++m)
#pragma unroll
        for (int l = 0; l < NE; ++l) du[m][l] = m == C ? 0.0f : float(cons[m][l] - cons[C][l]);
      T dm[NE], dp[NE];
      if constexpr (ALP_FAST && W == 6 && C == 2) {
        // both sides of every characteristic field in packed f32x2 arithmetic
        // the projection of cells (0, 5) and (1, 4) packed as well; cell 2 is
        // the face's left cell, whose increment is zero
        float2 chp[NE], out[NE];
#pragma unroll
        for (int n = 0; n < NE; ++n) {
          T L[NE];
          left_row<DIM, DIR, T>(n, r, L);
          float2 P0 = make_float2(0.0f, 0.0f), P1 = P0;
          float u3 = 0.0f;
          bool first = true;
#pragma unroll
          for (int q = 0; q < NE; ++q) {
            int const l = sum_seq<DIM, DIR>(q);
            if (!left_nonzero<DIM, DIR>(n, l)) continue;
            float2 const Ld = dup2(L[l]);
            float2 const a0 = make_float2(du[0][l], du[5][l]);
            float2 const a1 = make_float2(du[1][l], du[4][l]);
            P0 = first ? mul2(Ld, a0) : fma2(Ld, a0, P0);
            P1 = first ? mul2(Ld, a1) : fma2(Ld, a1, P1);
            u3 = fmaf(L[l], du[3][l], u3);
            first = false;
          }
          chp[n] = weno5_packed(P0, P1, make_float2(0.0f, u3), make_float2(u3, 0.0f),
                                make_float2(P1.y, P1.x));
        }
        to_physical_packed<DIM, DIR>(r, chp, out);
#pragma unroll
        for (int f = 0; f < NE; ++f) {
          dm[f] = out[f].x;
          dp[f] = out[f].y;
        }
      } else {
#pragma unroll
        for (int n = 0; n < NE; ++n) {
          T L[NE];
          left_row<DIM, DIR, T>(n, r, L);
          T uc[W];
#pragma unroll
          for (int m = 0; m < W; ++m) {
            T s = T(0);
#pragma unroll
            for (int q = 0; q < NE; ++q) {
              int const l = sum_seq<DIM, DIR>(q);
              if (!left_nonzero<DIM, DIR>(n, l)) continue;
              s = fmaf(L[l], du[m][l], s);
            }
            uc[m] = s;
          }
          weno5_pair(uc, ch[0][n], ch[1][n]);
        }
        to_physical<DIM, DIR, T>(r, ch[0], dm);
        to_physical<DIM, DIR, T>(r, ch[1], dp);
      }
      double cm[NE], cp[NE];
#pragma unroll
      for (int f = 0; f < NE; ++f) {
        cm[f] = cons[C][f] + double(dm[f]);
        cp[f] = cons[C][f] + double(dp[f]);
      }
      if (!(cm[MASS] > DBL_EPSILON) || !(cp[MASS] > DBL_EPSILON)) valid = false;
      double const one_l = inv(cm[MASS]), one_r = inv(cp[MASS]);
      double const pm = eos_pressure<DIM>(eos, cm[MASS], cm[MOMX], DIM > 1 ? cm[MOMX + (DIM > 1)] : 0.0,
                                          DIM > 2 ? cm[MOMX + 2 * (DIM > 2)] : 0.0, cm[ENERGY], one_l);
      double const pp = eos_pressure<DIM>(eos, cp[MASS], cp[MOMX], DIM > 1 ? cp[MOMX + (DIM > 1)] : 0.0,
                                          DIM > 2 ? cp[MOMX + 2 * (DIM > 2)] : 0.0, cp[ENERGY], one_r);
      if (!(pm > -B) || !(pp > -B)) valid = false;
      hllc_mixed<DIM, DIR>(eos, cm, cp, pm, pp, cm[mP] * one_l, cp[mP] * one_r, one_l, one_r, fd);
      return valid;
    } else if constexpr (SCHEME == FV_CHAR) {
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        T L[NE];
        left_row<DIM, DIR, T>(n, r, L);
        T uc[W];
#pragma unroll
        for (int m = 0; m < W; ++m) {
          T s = T(0);
          bool first = true;
#pragma unroll
          for (int q = 0; q < NE; ++q) {
            int const l = sum_seq<DIM, DIR>(q);
            if (!left_nonzero<DIM, DIR>(n, l)) continue;
            T const prod = L[l] * T(cons[m][l]);
            s = first ? prod : s + prod;
            first = false;
          }
          uc[m] = s;
        }
        pol.pair(uc, ch[0][n], ch[1][n]);
      }
      T cm[NE], cp[NE];
      to_physical<DIM, DIR, T>(r, ch[0], cm);
      to_physical<DIM, DIR, T>(r, ch[1], cp);
      if (!(cm[MASS] > eps_of<T>()) || !(cp[MASS] > eps_of<T>())) valid = false;
      // prime states of the reconstructed states (prime_state_handler.h:277-371),
      // pressure recovered in double
      T const one_l = inv(cm[MASS]), one_r = inv(cp[MASS]);
      double const pm = eos_pressure<DIM>(eos, double(cm[MASS]), double(cm[MOMX]),
                                          DIM > 1 ? double(cm[MOMX + (DIM > 1)]) : 0.0,
                                          DIM > 2 ? double(cm[MOMX + 2 * (DIM > 2)]) : 0.0,
                                          double(cm[ENERGY]), double(one_l));
      double const pp = eos_pressure<DIM>(eos, double(cp[MASS]), double(cp[MOMX]),
                                          DIM > 1 ? double(cp[MOMX + (DIM > 1)]) : 0.0,
                                          DIM > 2 ? double(cp[MOMX + 2 * (DIM > 2)]) : 0.0,
                                          double(cp[ENERGY]), double(one_r));
      if (!(pm > -B) || !(pp > -B)) valid = false;
      T const vl = cm[mP] * one_l;
      T const vr = cp[mP] * one_r;
      pol.template riemann<DIM, DIR, T>(eos, cm, cp, T(pm), T(pp), vl, vr, one_l, one_r, flux);
    } else {
      // Roe flux-vector splitting (flux_splitting_scheme.cpp:42-76, 185-315)
      double advd[W][NE];
#pragma unroll
      for (int m = 0; m < W; ++m) {
        double const one_rho = inv(cons[m][MASS]);
        double const p = eos_pressure<DIM>(
            eos, cons[m][MASS], cons[m][MOMX], DIM > 1 ? cons[m][MOMX + (DIM > 1)] : 0.0,
            DIM > 2 ? cons[m][MOMX + 2 * (DIM > 2)] : 0.0, cons[m][ENERGY], one_rho);
        double const vel = cons[m][mP] * one_rho;
        double const rho = cons[m][MASS];
        // the fast build uses rho u = m for the mass and momentum fluxes
        advd[m][MASS] = ALP_FAST ? cons[m][mP] : rho * vel;
        advd[m][ENERGY] = (cons[m][ENERGY] + p) * vel;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          double const vd = cons[m][MOMX + d] * one_rho;
          double v = ALP_FAST ? cons[m][mP] * vd : rho * (vel * vd);
          if (d == DIR) v += p;
          advd[m][MOMX + d] = v;
        }
      }
      T ev_nl0, ev_lin, ev_nl1;
      pol.template fs_eigenvalues<DIM, DIR, T>(eos, r, pt, pn, ev_nl0, ev_lin, ev_nl1);
      // FP32 form: increments against the face's left cell; the characteristic
      // flux of that cell, L f_i, is restored by R as f_i in double
      constexpr bool DELTA = sizeof(T) == 4;
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        T L[NE];
        left_row<DIM, DIR, T>(n, r, L);
        T const alpha = n == 0 ? ev_nl0 : (n == NE - 1 ? ev_nl1 : ev_lin);
        T pos[W], neg[W];
#pragma unroll
        for (int m = 0; m < W; ++m) {
          T sp = T(0), sn = T(0);
          bool first = true;
          if constexpr (DELTA && ALP_FAST) {
            // state and flux projections as the two lanes of packed f32x2
            // arithmetic: (L u, L f) += L[l] (du, df)
            float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int q = 0; q < NE; ++q) {
              int const l = sum_seq<DIM, DIR>(q);
              if (!left_nonzero<DIM, DIR>(n, l)) continue;
              float2 const d = make_float2(float(cons[m][l] - cons[C][l]),
                                           float(advd[m][l] - advd[C][l]));
              acc = first ? mul2(d, dup2(L[l])) : fma2(d, dup2(L[l]), acc);
              first = false;
            }
            pos[m] = fmaf(alpha, acc.x, acc.y);
            neg[m] = fmaf(-alpha, acc.x, acc.y);
            continue;
          }
#pragma unroll
          for (int q = 0; q < NE; ++q) {
            int const l = sum_seq<DIM, DIR>(q);
            if (!left_nonzero<DIM, DIR>(n, l)) continue;
            T const uct = (DELTA ? T(cons[m][l] - cons[C][l]) : T(cons[m][l])) * L[l];
            T const act = (DELTA ? T(advd[m][l] - advd[C][l]) : T(advd[m][l])) * L[l];
            if constexpr (ALP_FAST) {
              // project state (into sp) and flux (into sn), split afterwards:
              // L (f +/- alpha u) = L f +/- alpha L u
              sp = first ? uct : sp + uct;
              sn = first ? act : sn + act;
            } else {
              T const tp = act + alpha * uct;
              T const tn = act - alpha * uct;
              sp = first ? tp : sp + tp;
              sn = first ? tn : sn + tn;
            }
            first = false;
          }
          if constexpr (ALP_FAST) {
            pos[m] = sn + alpha * sp;
            neg[m] = sn - alpha * sp;
          } else {
            pos[m] = sp;
            neg[m] = sn;
          }
        }
        T wl, wr;
        pol.two(pos, neg, wl, wr);
        ch[0][n] = T(0.5) * (wl + wr);
      }
      to_physical<DIM, DIR, T>(r, ch[0], flux);
      if constexpr (DELTA) {
#pragma unroll
        for (int f = 0; f < NE; ++f) fd[f] = advd[C][f] + double(flux[f]);
        return valid;
      }
    }
  } else {
    // FV primitive reconstruction (primitive_state_reconstruction.h:56-107)
    double prim[W][NE];
#pragma unroll
    for (int m = 0; m < W; ++m) {
      prim[m][RHO] = cons[m][MASS];
      double const one_rho = inv(cons[m][MASS]);
#pragma unroll
      for (int d = 0; d < DIM; ++d) prim[m][VELX + d] = cons[m][MOMX + d] * one_rho;
      prim[m][PRES] = eos_pressure<DIM>(
          eos, cons[m][MASS], cons[m][MOMX], DIM > 1 ? cons[m][MOMX + (DIM > 1)] : 0.0,
          DIM > 2 ? cons[m][MOMX + 2 * (DIM > 2)] : 0.0, cons[m][ENERGY], one_rho);
    }
    if constexpr (sizeof(T) == 4) {
      // FP32 form: WENO5 of the increments against the left cell's primes
      double pmd[NE], ppd[NE];
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        T arr[W];
#pragma unroll
        for (int m = 0; m < W; ++m) arr[m] = T(prim[m][n] - prim[C][n]);
        T wl, wr;
        weno5_pair(arr, wl, wr);
        pmd[n] = prim[C][n] + double(wl);
        ppd[n] = prim[C][n] + double(wr);
      }
      double cm[NE], cp[NE];
      cm[MASS] = pmd[RHO];
      cp[MASS] = ppd[RHO];
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        cm[MOMX + d] = pmd[VELX + d] * pmd[RHO];
        cp[MOMX + d] = ppd[VELX + d] * ppd[RHO];
      }
      cm[ENERGY] = eos_energy<DIM, double>(eos, pmd[RHO], pmd[VELX], DIM > 1 ? pmd[VELX + (DIM > 1)] : 0.0,
                                           DIM > 2 ? pmd[VELX + 2 * (DIM > 2)] : 0.0, pmd[PRES]);
      cp[ENERGY] = eos_energy<DIM, double>(eos, ppd[RHO], ppd[VELX], DIM > 1 ? ppd[VELX + (DIM > 1)] : 0.0,
                                           DIM > 2 ? ppd[VELX + 2 * (DIM > 2)] : 0.0, ppd[PRES]);
      if (!(cm[MASS] > DBL_EPSILON) || !(cp[MASS] > DBL_EPSILON)) valid = false;
      if (!(pmd[PRES] > -B) || !(ppd[PRES] > -B)) valid = false;
      hllc_mixed<DIM, DIR>(eos, cm, cp, pmd[PRES], ppd[PRES], pmd[VELX + DIR], ppd[VELX + DIR],
                           inv(cm[MASS]), inv(cp[MASS]), fd);
      return valid;
    } else {
      T pm[NE], pp[NE];
#pragma unroll
      for (int n = 0; n < NE; ++n) {
        T arr[W];
#pragma unroll
        for (int m = 0; m < W; ++m) arr[m] = T(prim[m][n]);
        pol.pair(arr, pm[n], pp[n]);
      }
      // PrimeStatesToConservatives (prime_state_handler.h:195-275)
      T cm[NE], cp[NE];
      cm[MASS] = pm[RHO];
      cp[MASS] = pp[RHO];
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        cm[MOMX + d] = pm[VELX + d] * pm[RHO];
        cp[MOMX + d] = pp[VELX + d] * pp[RHO];
      }
      cm[ENERGY] = eos_energy<DIM, T>(eos, pm[RHO], pm[VELX], DIM > 1 ? pm[VELX + (DIM > 1)] : T(0),
                                      DIM > 2 ? pm[VELX + 2 * (DIM > 2)] : T(0), pm[PRES]);
      cp[ENERGY] = eos_energy<DIM, T>(eos, pp[RHO], pp[VELX], DIM > 1 ? pp[VELX + (DIM > 1)] : T(0),
                                      DIM > 2 ? pp[VELX + 2 * (DIM > 2)] : T(0), pp[PRES]);
      if (!(cm[MASS] > eps_of<T>()) || !(cp[MASS] > eps_of<T>())) valid = false;
      if (!(double(pm[PRES]) > -B) || !(double(pp[PRES]) > -B)) valid = false;
      // HLLC's own 1/density (hllc_riemann_solver.h:75-78)
      pol.template riemann<DIM, DIR, T>(eos, cm, cp, pm[PRES], pp[PRES], pm[VELX + DIR], pp[VELX + DIR],
                        inv(cm[MASS]), inv(cp[MASS]), flux);
    }
  }

#pragma unroll
  for (int f = 0; f < NE; ++f) fd[f] = double(flux[f]);
  return valid;
}

}  // namespace alp
