// Stage-update, signal-speed and time-step arithmetic shared by every stepping
// kernel (kernels.cu, tile_step.cu): one definition of each expression, so the
// fused tile kernel and the face-flux + stage-update kernels round alike.
#pragma once

#include <cfloat>

#include "layout.cuh"
#include "numerics.cuh"

namespace alp {

namespace {
// Stage coefficients: indices 0-2 the SSP-RK3 stages (runge_kutta_3_TVD.h:
// 41-59), 3-4 the TVD-RK2 stages (runge_kutta_2_TVD.h:37-56); per stage the
// multiplier of dt and the buffer multipliers of the stage input and of the
// step's initial state (unused in a first stage). Uout = a0 U + a1 U0 +
// c dt RHS (time_integrator.h:98-113, 434-457).
__constant__ double kRkC[5] = {1.0, 0.25, 2.0 / 3.0, 1.0, 0.5};
__constant__ double kRkA0[5] = {0.0, 0.25, 2.0 / 3.0, 0.0, 0.5};
__constant__ double kRkA1[5] = {0.0, 0.75, 1.0 / 3.0, 0.0, 0.5};
}  // namespace

__host__ __device__ constexpr bool rk_first_stage(int stage) { return stage == 0 || stage == 3; }

// The coefficients of one stage with the case's dt folded in.
struct RkStage {
  double a0, a1, cdt;
  bool first;
};
__device__ __forceinline__ RkStage rk_stage(int stage, double dt) {
  return RkStage{kRkA0[stage], kRkA1[stage], kRkC[stage] * (0.0 + dt), rk_first_stage(stage)};
}
// Stage output of one cell and field; u0 is not read in a first stage.
__device__ __forceinline__ double rk_apply(RkStage const &r, double uin, double u0, double rhs) {
  double u = uin;
  if (!r.first) u = r.a0 * u + r.a1 * u0;
  return u + r.cdt * rhs;
}

// SpaceSolver flux divergence of one cell and field (space_solver.cpp:131-153):
// DimensionAwareConsistencyManagedSum(dFx, dFy, dFz) * (1 / cell size), each
// difference the cell's low face minus its high face.
template <int DIM>
__device__ __forceinline__ double flux_divergence(double fx_lo, double fx_hi, double fy_lo,
                                                  double fy_hi, double fz_lo, double fz_hi,
                                                  double one_cell_size) {
  double const dx = fx_lo - fx_hi;
  double dy = 0.0, dz = 0.0;
  if constexpr (DIM > 1) dy = fy_lo - fy_hi;
  if constexpr (DIM > 2) dz = fz_lo - fz_hi;
  return dacms<DIM>(dx, dy, dz) * one_cell_size;
}

// Flux divergence of interior cell (i, j, k) of one field from the reference
// flux arrays of the three directions (Fx, Fy, Fz at the field's offset).
template <int DIM>
__device__ __forceinline__ double divergence(double const *Fx, double const *Fy,
                                             double const *Fz, int i, int j, int k,
                                             double one_cell_size) {
  using G = Geo<DIM>;
  return flux_divergence<DIM>(Fx[G::face(i, j + 1, k + 1)], Fx[G::face(i + 1, j + 1, k + 1)],
                              DIM > 1 ? Fy[G::face(i + 1, j, k + 1)] : 0.0,
                              DIM > 1 ? Fy[G::face(i + 1, j + 1, k + 1)] : 0.0,
                              DIM > 2 ? Fz[G::face(i + 1, j + 1, k)] : 0.0,
                              DIM > 2 ? Fz[G::face(i + 1, j + 1, k + 1)] : 0.0, one_cell_size);
}

// Interior cell (i, j, k) of thread t of a block's 16^DIM cells (z fastest).
template <int DIM>
__host__ __device__ __forceinline__ void interior_coords(int t, int &i, int &j, int &k) {
  if constexpr (DIM == 3) {
    i = t >> 8;
    j = (t >> 4) & 15;
    k = t & 15;
  } else if constexpr (DIM == 2) {
    i = t >> 4;
    j = t & 15;
    k = 0;
  } else {
    i = t;
    j = 0;
    k = 0;
  }
}

// Stage update of interior cell t of the block in `slot`, every field: the flux
// divergence from the block's face-flux arrays Fb (directions dstride apart)
// and the RK stage into Uout. Every stage update computes it this way.
template <int DIM>
__device__ __forceinline__ void stage_update_cell(double const *Uin, double const *U0, double *Uout,
                                                  double const *Fb, long long dstride, int slot,
                                                  int t, double one_cell_size, RkStage const &rk) {
  using G = Geo<DIM>;
  int i, j, k;
  interior_coords<DIM>(t, i, j, k);
  int const c = G::cell(i + G::fic(0), j + G::fic(1), k + G::fic(2));
  size_t const base = (size_t)slot * G::BLOCK_DOUBLES + c;
#pragma unroll
  for (int f = 0; f < G::NE; ++f) {
    double const *fx = Fb + f * G::FACES;
    double const rhs = 0.0 + divergence<DIM>(fx, fx + dstride, fx + 2 * dstride, i, j, k,
                                             one_cell_size);
    size_t const x = base + (size_t)f * G::CELLS;
    Uout[x] = rk_apply(rk, Uin[x], rk.first ? 0.0 : U0[x], rhs);
  }
}

__device__ __forceinline__ unsigned ld_acquire_u32(unsigned const *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits (one thread of a CTA) until *c reaches `target`, bounded: 2^22 polls
// (a second or two of L2 round trips). On running out it sets *err and
// returns false; a wait that finds *err set gives up within 1024 polls.
__device__ __forceinline__ bool wait_count(unsigned const *c, unsigned target, int *err) {
  for (int i = 0; i < (1 << 22); ++i) {
    if (ld_acquire_u32(c) >= target) return true;
    if ((i & 1023) == 1023 && *reinterpret_cast<int volatile *>(err)) return false;
  }
  if (ld_acquire_u32(c) >= target) return true;
  atomicOr(err, 1);
  return false;
}

// Signal speed of one cell for ComputeTimestepSize
// (modular_algorithm_assembler.cpp:1840-1870): ConsistencyManagedSum(|u_d| + c).
// Sets bad for a NaN, a non-positive density or an imaginary sound speed.
template <int DIM>
__device__ __forceinline__ double cell_signal_speed(Eos const &eos, double const (&c)[DIM + 2],
                                                    int &bad) {
  double const one_density = inv(c[MASS]);
  double const p = eos_pressure<DIM>(eos, c[MASS], c[MOMX], DIM > 1 ? c[MOMX + (DIM > 1)] : 0.0,
                                     DIM > 2 ? c[MOMX + 2 * (DIM > 2)] : 0.0, c[ENERGY],
                                     one_density);
  double const cs = eos_speed_of_sound<double>(eos, c[MASS], p, one_density);
  double v[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < DIM; ++d) v[d] = fabs(c[MOMX + d] * one_density) + cs;
  double s;
  if constexpr (DIM == 1) s = v[0];
  else if constexpr (DIM == 2) s = v[0] + v[1];
  else s = cms3(v[0], v[1], v[2]);
  if (!(s >= 0.0) || !(c[MASS] > 0.0)) bad = 1;
  return s;
}

// dt = CFL / (smax / dx_finest), clipped to the end time
// (modular_algorithm_assembler.cpp:1932, 1961-1982); 0 once t >= t_end, the
// step budget is spent, the case stopped or is held, which makes every kernel
// skip the case. Consumes smax (reset to 0 for the next reduction).
__device__ __forceinline__ void case_dt_finalize(CaseState &s) {
  double const smax = __longlong_as_double((long long)s.smax_bits);
  s.smax_bits = 0ull;
  double dt = smax / s.h_min;
  double local = dt == 0.0 ? DBL_MAX : s.cfl / dt;
  if (s.t + local > s.t_end) local = dmax(s.t_end - s.t, 0.0);
  if (!(s.t < s.t_end)) local = 0.0;
  if (s.max_steps > 0 && s.steps >= s.max_steps) local = 0.0;
  if (s.status || s.hold) local = 0.0;
  s.dt = local;
}

// t += dt, steps += 1 for a case that stepped (dt > 0).
__device__ __forceinline__ void case_commit(CaseState &s) {
  if (s.dt > 0.0) {
    s.t = s.t + (0.0 + s.dt);
    s.steps += 1;
  }
}

}  // namespace alp
