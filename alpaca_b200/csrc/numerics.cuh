// Device numerics of the ALPACA face flux: stiffened-gas EOS, WENO5-JS, the
// Roe eigensystem, HLLC with Einfeldt speeds and Roe flux-vector splitting.
// Each function states the reference lines (ALPACA src/) whose arithmetic it
// follows; the association order of every sum is kept so that results agree
// with the CPU reference to rounding (FMA contraction is the only difference).
// T is the compute type of reconstruction and flux (double, or float in the
// FP32-flux form); pressure recovery from total energy always runs in double.
//
// Two builds share this file. The strict build (ALP_STRICT, compiled with
// -fmad=false) evaluates every expression exactly as the reference writes it,
// IEEE division included, and reproduces the reference bit for bit. The fast
// build replaces divisions by Newton-refined reciprocals (reused where the same
// divisor recurs), evaluates the WENO5 weights of a face's two reconstructions
// with shared second differences and one reciprocal, and takes float square
// roots from the hardware approximation; all change results only at the
// rounding level.
#pragma once

#include <cfloat>

#include "layout.cuh"

#ifdef ALP_STRICT
#define ALP_FAST 0
#else
#define ALP_FAST 1
#endif

namespace alp {

// Reciprocal by Newton-Raphson iteration on f(y) = 1/y - b (y <- y + y(1 - b y)),
// seeded with the PTX approximate reciprocal; two iterations take the seed's
// ~2^-20 relative error below one ulp.
__device__ __forceinline__ double rcp_nr(double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  return y;
}

// 1/sqrt(x) by Newton-Raphson iteration on f(y) = 1/y^2 - x
// (y <- y + y (1 - x y^2) / 2), seeded with the PTX approximate reciprocal
// square root; each iteration squares the relative error, two take it below
// the rounding of the last steps (fast build only).
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x * y, y, 1.0);
  y = fma(0.5 * y, e, y);
  e = fma(-x * y, y, 1.0);
  y = fma(0.5 * y, e, y);
  return y;
}

// 1/x: IEEE division in the strict build, rcp_nr (double) or the PTX
// approximate reciprocal (float, one instruction, about 1 ulp) in the fast
// build.
__device__ __forceinline__ double inv(double x) {
  if constexpr (ALP_FAST) return rcp_nr(x);
  else return 1.0 / x;
}
__device__ __forceinline__ float inv(float x) {
  if constexpr (ALP_FAST) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
  } else {
    return 1.0f / x;
  }
}
// a / b, where ib is 1/b as returned by inv(b): the strict build divides.
template <typename T> __device__ __forceinline__ T quot(T a, T b, T ib) {
  if constexpr (ALP_FAST) return a * ib;
  else return a / b;
}
template <typename T> __device__ __forceinline__ T quot(T a, T b) {
  if constexpr (ALP_FAST) return a * inv(b);
  else return a / b;
}

// Square root: IEEE in double and in the strict build; in the fast build's
// float arithmetic (the FP32-flux form) the PTX approximate square root, one
// instruction with a few ulp of error against the IEEE sequence.
__device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float tsqrt(float x) {
  if constexpr (ALP_FAST) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
  } else {
    return sqrtf(x);
  }
}

// A product rounded on its own (never fused into a following addition).
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }

template <typename T> __device__ __forceinline__ T dmin(T a, T b) { return (b < a) ? b : a; }
template <typename T> __device__ __forceinline__ T dmax(T a, T b) { return (a < b) ? b : a; }
template <typename T> __device__ __forceinline__ T eps_of();
template <> __device__ __forceinline__ double eps_of<double>() { return DBL_EPSILON; }
template <> __device__ __forceinline__ float eps_of<float>() { return FLT_EPSILON; }

// ConsistencyManagedSum with FUSY on (utilities/mathematical_functions.h:79-89)
template <typename T> __device__ __forceinline__ T cms3(T a, T b, T c) {
  T const s1 = (a + b) + c;
  T const s2 = (a + c) + b;
  T const s3 = (b + c) + a;
  T mn = s1, mx = s1;
  if (s2 < mn) mn = s2;
  if (s3 < mn) mn = s3;
  if (mx < s2) mx = s2;
  if (mx < s3) mx = s3;
  return T(0.5) * (mn + mx);
}

// DimensionAwareConsistencyManagedSum (mathematical_functions.h:98-108)
template <int DIM, typename T> __device__ __forceinline__ T dacms(T a, T b, T c) {
  if constexpr (DIM == 1) return a;
  else if constexpr (DIM == 2) return a + b;
  else return cms3(a, b, c);
}

// Sum of three squares, independent of the order of its terms as the
// consistency-managed sum is. The fast build sorts them (the bit patterns of
// non-negative floating-point values order like the values) and adds the two
// smaller first: two additions and integer compares instead of seven
// additions and four floating-point compares. The strict build and 1D/2D keep
// DimensionAwareConsistencyManagedSum.
template <int DIM, typename T> __device__ __forceinline__ T sum_sq(T a, T b, T c) {
  if constexpr (!ALP_FAST || DIM < 3) {
    return dacms<DIM>(a, b, c);
  } else if constexpr (sizeof(T) == 8) {
    long long const ia = __double_as_longlong(a), ib = __double_as_longlong(b);
    long long const ic = __double_as_longlong(c);
    long long const lo = min(ia, ib), hi = max(ia, ib);
    long long const x0 = min(lo, ic), t = max(lo, ic);
    long long const x1 = min(t, hi), x2 = max(t, hi);
    return (__longlong_as_double(x0) + __longlong_as_double(x1)) + __longlong_as_double(x2);
  } else {
    int const ia = __float_as_int(a), ib = __float_as_int(b), ic = __float_as_int(c);
    int const lo = min(ia, ib), hi = max(ia, ib);
    int const x0 = min(lo, ic), t = max(lo, ic);
    int const x1 = min(t, hi), x2 = max(t, hi);
    return (__int_as_float(x0) + __int_as_float(x1)) + __int_as_float(x2);
  }
}

// ---- stiffened gas (generic_stiffened_gas.h:40-102, stiffened_gas.cpp:62-149,
//      stiffened_gas_safe.cpp:61-146) --------------------------------------

struct Eos {
  double gamma, B;
  int safe;
};

// one_mass = inv(mass) (unused by the strict build, which divides)
template <int DIM>
__device__ __forceinline__ double eos_pressure(Eos const &e, double mass, double mx, double my,
                                               double mz, double energy, double one_mass) {
  if (e.safe) {
    double const m = dmax(mass, DBL_EPSILON);
    double const p =
        -e.gamma * e.B +
        (e.gamma - 1.0) * (energy - quot(0.5 * sum_sq<DIM>(mx * mx, my * my, mz * mz), m,
                                         mass > DBL_EPSILON ? one_mass : inv(m)));
    return dmax(p, -e.B + DBL_EPSILON);
  }
  double const q = 0.5 * sum_sq<DIM>(mx * mx, my * my, mz * mz);
  return -e.gamma * e.B + (e.gamma - 1.0) * (energy - quot(q, mass, one_mass));
}
template <int DIM>
__device__ __forceinline__ double eos_pressure(Eos const &e, double mass, double mx, double my,
                                               double mz, double energy) {
  return eos_pressure<DIM>(e, mass, mx, my, mz, energy, ALP_FAST ? inv(mass) : 0.0);
}

template <int DIM, typename T>
__device__ __forceinline__ T eos_energy(Eos const &e, T rho, T u, T v, T w, T p) {
  T const g = T(e.gamma), B = T(e.B);
  return quot(p + g * B, g - T(1)) + (T(0.5) * sum_sq<DIM>(u * u, v * v, w * w) * rho);
}

// one_rho = inv(rho) (unused by the strict build)
template <typename T>
__device__ __forceinline__ T eos_speed_of_sound(Eos const &e, T rho, T p, T one_rho) {
  T const g = T(e.gamma), B = T(e.B);
  if (e.safe) {
    T const r = dmax(rho, eps_of<T>());
    T const c2 = quot(g * (p + B), r, rho > eps_of<T>() ? one_rho : inv(r));
    return tsqrt(dmax(c2, eps_of<T>()));
  }
  return tsqrt(quot(g * (p + B), rho, one_rho));
}
template <typename T> __device__ __forceinline__ T eos_speed_of_sound(Eos const &e, T rho, T p) {
  return eos_speed_of_sound<T>(e, rho, p, ALP_FAST ? inv(rho) : T(0));
}

// ---- WENO5-JS (stencils/spatial_reconstruction_stencils/weno5.h:88-158) --
// a[0..5] are cells i-2..i+3 around face i+1/2; UpwindLeft uses {offset 0,
// sign +1}, UpwindRight {1, -1} (stencils/apply_wrapper.h:47-57).
template <typename T>
__device__ __forceinline__ T weno5_core(T v1, T v2, T v3, T v4, T v5) {
  T const c1 = T(13.0 / 12.0), c2 = T(0.25);
  T const s11 = v1 + T(-2.0) * v2 + v3;
  T const s12 = v1 + T(-4.0) * v2 + T(3.0) * v3;
  T const s1 = c1 * s11 * s11 + c2 * s12 * s12;
  T const s21 = v2 + T(-2.0) * v3 + v4;
  T const s22 = v2 + T(-1.0) * v4;
  T const s2 = c1 * s21 * s21 + c2 * s22 * s22;
  T const s31 = v3 + T(-2.0) * v4 + v5;
  T const s32 = T(3.0) * v3 + T(-4.0) * v4 + v5;
  T const s3 = c1 * s31 * s31 + c2 * s32 * s32;
  T const eps = T(1.0e-6);
  T const q1 = T(2.0 / 6.0) * v1 + T(-7.0 / 6.0) * v2 + T(11.0 / 6.0) * v3;
  T const q2 = T(-1.0 / 6.0) * v2 + T(5.0 / 6.0) * v3 + T(2.0 / 6.0) * v4;
  T const q3 = T(2.0 / 6.0) * v3 + T(5.0 / 6.0) * v4 + T(-1.0 / 6.0) * v5;
  T const t1 = (s1 + eps) * (s1 + eps);
  T const t2 = (s2 + eps) * (s2 + eps);
  T const t3 = (s3 + eps) * (s3 + eps);
  if constexpr (ALP_FAST && sizeof(T) == 8) {
    // alpha_k = d_k / t_k scaled by t1 t2 t3: one reciprocal instead of four
    // divisions (t_k >= 1e-12 and the products stay far inside the double range)
    T const b1 = T(0.1) * (t2 * t3);
    T const b2 = T(0.6) * (t1 * t3);
    T const b3 = T(0.3) * (t1 * t2);
    return (b1 * q1 + b2 * q2 + b3 * q3) * inv(b1 + b2 + b3);
  } else {
    T const a1 = quot(T(0.1), t1);
    T const a2 = quot(T(0.6), t2);
    T const a3 = quot(T(0.3), t3);
    T const one_a_sum = quot(T(1.0), a1 + a2 + a3);
    T const w1 = a1 * one_a_sum;
    T const w2 = a2 * one_a_sum;
    T const w3 = a3 * one_a_sum;
    return w1 * q1 + w2 * q2 + w3 * q3;
  }
}
template <typename T> __device__ __forceinline__ T weno5_left(T const (&a)[6]) {
  return weno5_core(a[0], a[1], a[2], a[3], a[4]);
}
template <typename T> __device__ __forceinline__ T weno5_right(T const (&a)[6]) {
  return weno5_core(a[5], a[4], a[3], a[2], a[1]);
}

// Fast-build WENO5-JS from first differences. For a stencil v1..v5 around
// the face of v3, with g1..g4 = v2-v1, v3-v2, v4-v3, v5-v4 and the second
// differences d1..d3 = g2-g1, g3-g2, g4-g3, the three candidate values are
//   q1 = v3 + (5 g2 - 2 g1) / 6, q2 = v3 + (g2 + 2 g3) / 6, q3 = v3 + (4 g3 - g4) / 6
// and the smoothness indicators, four times larger with eps four times larger
// (every (beta + eps)^2 scaled alike, so the weights do not change),
//   13/3 d_k^2 + e_k^2 with e = 3 g2 - g1, g2 + g3, g4 - 3 g3.
// The ideal weights 0.1, 0.6, 0.3 enter as 1, 6, 3. The result is
// v3 + num / (6 den); passing the differences of the mirrored stencil without
// their sign change (g_k' = -g) negates num and leaves den unchanged.
// alpha_k scaled by t1 t2 t3 (no reciprocal here). In float the t_k are first
// multiplied by the power of two that brings the largest into [1, 2) (exact:
// the scale is built from the exponent bits), so the products stay inside the
// float range; a product that underflows belongs to a weight below 2^-126 of
// the largest.
template <typename T> struct Weno5Frac { T num, den; };

template <typename T>
__device__ __forceinline__ Weno5Frac<T> weno5_frac(T g1, T g2, T g3, T g4, T d1, T d2, T d3) {
  T const c = T(13.0 / 3.0);
  T const e1 = T(3.0) * g2 - g1;
  T const e2 = g2 + g3;
  T const e3 = g4 + T(-3.0) * g3;
  T const eps = T(4.0e-6);
  T const s1 = (c * d1) * d1 + (e1 * e1 + eps);
  T const s2 = (c * d2) * d2 + (e2 * e2 + eps);
  T const s3 = (c * d3) * d3 + (e3 * e3 + eps);
  T const t1 = s1 * s1, t2 = s2 * s2, t3 = s3 * s3;
  T const r1 = T(5.0) * g2 + T(-2.0) * g1;
  T const r2 = g2 + T(2.0) * g3;
  T const r3 = T(4.0) * g3 - g4;
  T u1 = t1, u2 = t2, u3 = t3;
  if constexpr (sizeof(T) == 4) {
    unsigned const e = min((__float_as_uint(fmaxf(t1, fmaxf(t2, t3))) >> 23) & 0xffu, 253u);
    float const sc = __uint_as_float((254u - e) << 23);
    u1 = t1 * sc;
    u2 = t2 * sc;
    u3 = t3 * sc;
  }
  T const b1 = u2 * u3;
  T const b2 = T(6.0) * (u1 * u3);
  T const b3 = T(3.0) * (u1 * u2);
  return {b1 * r1 + b2 * r2 + b3 * r3, b1 + b2 + b3};
}

// v_l + num_l / (6 den_l) and v_r - num_r / (6 den_r). Double: one reciprocal
// of the product of the two denominators (each between ~1e-22 and ~1e7 |g|^8,
// so the product stays in range for differences up to ~1e17). Float: one
// reciprocal per side (a scaled denominator can be as small as the ratio of two
// smoothness terms, so the product of two could underflow).
template <typename T>
__device__ __forceinline__ void weno5_finish(T v_l, Weno5Frac<T> const &l, T v_r,
                                             Weno5Frac<T> const &r, T &left, T &right) {
  if constexpr (sizeof(T) == 8) {
    T const rr = inv((T(6.0) * l.den) * r.den);
    left = v_l + l.num * (r.den * rr);
    right = v_r - r.num * (l.den * rr);
  } else {
    left = v_l + l.num * inv(T(6.0) * l.den);
    right = v_r - r.num * inv(T(6.0) * r.den);
  }
}

// ---- packed FP32 pairs (Blackwell f32x2: one instruction for two lanes) ----
// Used by the fast build's FP32-flux form, where both sides of a face run the
// same arithmetic: lane x the left (UpwindLeft) side, lane y the right one.
__device__ __forceinline__ float2 dup2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b, rounded once (a + (-1) b)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, dup2(-1.0f), a); }

// UpwindLeft and UpwindRight of one face, packed: P_k = (a[k], a[5-k]) for
// k = 0 .. 4 of the six cells a[0..5] (i-2 .. i+3). Lane y runs the mirrored
// stencil, whose first differences are the negated ones weno5_frac takes for
// the right side, so both lanes end as P_2 + num / (6 den) (weno5_frac; the
// second differences and the e_k enter squared, so their signs do not matter).
__device__ __forceinline__ float2 weno5_packed(float2 P0, float2 P1, float2 P2, float2 P3,
                                               float2 P4) {
  float2 const ng1 = sub2(P0, P1), g2 = sub2(P2, P1), g3 = sub2(P3, P2), ng4 = sub2(P3, P4);
  float2 const d1 = add2(g2, ng1), d2 = sub2(g3, g2), d3 = add2(ng4, g3);
  float2 const e1 = fma2(dup2(3.0f), g2, ng1);
  float2 const e2 = add2(g2, g3);
  float2 const e3 = fma2(dup2(3.0f), g3, ng4);
  float2 const c = dup2(13.0f / 3.0f), eps = dup2(4.0e-6f);
  float2 const s1 = fma2(mul2(c, d1), d1, fma2(e1, e1, eps));
  float2 const s2 = fma2(mul2(c, d2), d2, fma2(e2, e2, eps));
  float2 const s3 = fma2(mul2(c, d3), d3, fma2(e3, e3, eps));
  float2 const t1 = mul2(s1, s1), t2 = mul2(s2, s2), t3 = mul2(s3, s3);
  float2 const r1 = fma2(dup2(2.0f), ng1, mul2(dup2(5.0f), g2));
  float2 const r2 = fma2(dup2(2.0f), g3, g2);
  float2 const r3 = fma2(dup2(4.0f), g3, ng4);
  // per lane: the power of two that brings the largest t_k into [1, 2)
  unsigned const ex = min((__float_as_uint(fmaxf(t1.x, fmaxf(t2.x, t3.x))) >> 23) & 0xffu, 253u);
  unsigned const ey = min((__float_as_uint(fmaxf(t1.y, fmaxf(t2.y, t3.y))) >> 23) & 0xffu, 253u);
  float2 const sc = make_float2(__uint_as_float((254u - ex) << 23), __uint_as_float((254u - ey) << 23));
  float2 const u1 = mul2(t1, sc), u2 = mul2(t2, sc), u3 = mul2(t3, sc);
  float2 const b1 = mul2(u2, u3);
  float2 const b2 = mul2(dup2(6.0f), mul2(u1, u3));
  float2 const b3 = mul2(dup2(3.0f), mul2(u1, u2));
  float2 const num = fma2(b3, r3, fma2(b2, r2, mul2(b1, r1)));
  float2 const q = mul2(dup2(6.0f), add2(add2(b1, b2), b3));
  return fma2(num, make_float2(inv(q.x), inv(q.y)), P2);
}

// UpwindLeft and UpwindRight of one face from the same six cells a[0..5]
// (i-2..i+3). The fast build shares the first differences and the second
// differences centred on a[2] and a[3] between the two (double), or runs the
// two sides as the lanes of packed f32x2 arithmetic (float).
template <typename T>
__device__ __forceinline__ void weno5_pair(T const (&a)[6], T &left, T &right) {
  if constexpr (!ALP_FAST) {
    left = weno5_left(a);
    right = weno5_right(a);
  } else if constexpr (sizeof(T) == 4) {
    float2 const r = weno5_packed(make_float2(a[0], a[5]), make_float2(a[1], a[4]),
                                  make_float2(a[2], a[3]), make_float2(a[3], a[2]),
                                  make_float2(a[4], a[1]));
    left = r.x;
    right = r.y;
  } else {
    T const G0 = a[1] - a[0], G1 = a[2] - a[1], G2 = a[3] - a[2], G3 = a[4] - a[3];
    T const G4 = a[5] - a[4];
    T const D1 = G1 - G0, D2 = G2 - G1, D3 = G3 - G2, D4 = G4 - G3;
    weno5_finish(a[2], weno5_frac(G0, G1, G2, G3, D1, D2, D3), a[3],
                 weno5_frac(G4, G3, G2, G1, D4, D3, D2), left, right);
  }
}

// UpwindLeft of a and UpwindRight of b (flux splitting: the positive and
// negative split fluxes).
template <typename T>
__device__ __forceinline__ void weno5_two(T const (&a)[6], T const (&b)[6], T &left, T &right) {
  if constexpr (!ALP_FAST) {
    left = weno5_left(a);
    right = weno5_right(b);
  } else if constexpr (sizeof(T) == 4) {
    // lane y: b mirrored
    float2 const r = weno5_packed(make_float2(a[0], b[5]), make_float2(a[1], b[4]),
                                  make_float2(a[2], b[3]), make_float2(a[3], b[2]),
                                  make_float2(a[4], b[1]));
    left = r.x;
    right = r.y;
  } else {
    T const A0 = a[1] - a[0], A1 = a[2] - a[1], A2 = a[3] - a[2], A3 = a[4] - a[3];
    T const B1 = b[2] - b[1], B2 = b[3] - b[2], B3 = b[4] - b[3], B4 = b[5] - b[4];
    weno5_finish(a[2], weno5_frac(A0, A1, A2, A3, A1 - A0, A2 - A1, A3 - A2), b[3],
                 weno5_frac(B4, B3, B2, B1, B4 - B3, B3 - B2, B2 - B1), left, right);
  }
}

// ---- Roe eigensystem (solvers/eigendecomposition.h:181-467) --------------
// The left/right eigenvector matrices are never stored: their entries are
// generated from the Roe-averaged scalars below when applied.
template <typename T> struct Roe {
  T up, u1, u2;     // principal, first and second minor velocity
  T H;              // enthalpy
  T c, cc, one_cc;  // speed of sound, c^2, 1/c^2
  T half_cc;        // 0.5 * one_cc
  T gru;            // Gruneisen coefficient gamma - 1
  T rho, one_rho;   // Roe density and its inverse
  T q2;             // |u|^2 (dimension-aware sum)
};

// minor directions (eigendecomposition.h:84-125)
template <int DIR> struct Minor;
template <> struct Minor<0> { static constexpr int m1 = 1, m2 = 2; };
template <> struct Minor<1> { static constexpr int m1 = 0, m2 = 2; };
template <> struct Minor<2> { static constexpr int m1 = 0, m2 = 1; };

// symmetry-preserving summation order of the characteristic projection
// (solvers/state_reconstruction/state_reconstruction.h:35-58): position q of
// the sequence for direction DIR.
template <int DIM, int DIR> __host__ __device__ constexpr int sum_seq(int q) {
  if (DIM == 1) return q == 0 ? MOMX : (q == 1 ? MASS : ENERGY);
  if (DIM == 2) return q < 2 ? MOMX + q : (q == 2 ? MASS : ENERGY);
  if (q >= 3) return q == 3 ? MASS : ENERGY;
  // 3D: X -> (MomY, MomZ, MomX), Y -> (MomZ, MomX, MomY), Z -> (MomX, MomY, MomZ)
  return MOMX + (DIR + 1 + q) % 3;
}

// Cell quantities the Roe average needs; conservatives are double.
template <int DIM, int DIR> struct CellPrims {
  double rho, one_rho, p, up, u1, u2, H;
};

template <int DIM, int DIR>
__device__ __forceinline__ CellPrims<DIM, DIR> cell_prims(Eos const &e, double const (&c)[DIM + 2]) {
  CellPrims<DIM, DIR> r;
  r.rho = c[MASS];
  r.one_rho = inv(c[MASS]);
  double const mx = c[MOMX];
  double const my = DIM > 1 ? c[MOMX + (DIM > 1 ? 1 : 0)] : 0.0;
  double const mz = DIM > 2 ? c[MOMX + (DIM > 2 ? 2 : 0)] : 0.0;
  // velocities from the prime-state buffer: momentum * (1/rho)
  // (prime_state_handler.h:293-311)
  r.up = c[MOMX + DIR] * r.one_rho;
  r.u1 = DIM > 1 ? c[MOMX + (DIM > 1 ? Minor<DIR>::m1 : 0)] * r.one_rho : 0.0;
  r.u2 = DIM > 2 ? c[MOMX + (DIM > 2 ? Minor<DIR>::m2 : 0)] * r.one_rho : 0.0;
  r.p = eos_pressure<DIM>(e, c[MASS], mx, my, mz, c[ENERGY], r.one_rho);
  // Enthalpy (stiffened_gas.cpp:88-96 / stiffened_gas_safe.cpp:77-84)
  r.H = e.safe ? quot(c[ENERGY] + r.p, dmax(c[MASS], DBL_EPSILON))
               : quot(c[ENERGY] + r.p, c[MASS], r.one_rho);
  return r;
}

// Roe averages of one face (eigendecomposition.h:252-310)
template <int DIM, int DIR, typename T>
__device__ __forceinline__ Roe<T> roe_average(Eos const &e, CellPrims<DIM, DIR> const &t,
                                              CellPrims<DIM, DIR> const &n) {
  Roe<T> r;
  T const gB = T(e.gamma * e.B);
  T const psi_t = (T(t.p) + gB) * T(t.one_rho);
  T const psi_n = (T(n.p) + gB) * T(n.one_rho);
  // sr_k * rho_div are the Roe weights sqrt(rho_k) / (sqrt(rho_t) + sqrt(rho_n))
  constexpr bool WEIGHTS = ALP_FAST && sizeof(T) == 8;
  T sr_t, sr_n, rho_div;
  if constexpr (WEIGHTS) {
    // the weights themselves (rho_div = 1) from one reciprocal square root:
    // mu = sqrt(rho_t / rho_n), lambda = 1 / mu, w_t = 1 / (1 + lambda),
    // w_n = lambda w_t, Roe density rho_t lambda and its inverse mu / rho_t
    T const ratio = n.rho * t.one_rho;
    T const mu = rsqrt_nr(ratio);
    T const lambda = ratio * mu;
    sr_t = inv(T(1) + lambda);
    sr_n = lambda * sr_t;
    rho_div = T(1);
    r.rho = t.rho * lambda;
    r.one_rho = t.one_rho * mu;
  } else {
    sr_t = tsqrt(T(t.rho));
    sr_n = tsqrt(T(n.rho));
    rho_div = quot(T(1), sr_t + sr_n);
    r.rho = sr_t * sr_n;
    r.one_rho = quot(T(1), r.rho);
  }
  r.up = ((T(t.up) * sr_t) + (T(n.up) * sr_n)) * rho_div;
  r.u1 = ((T(t.u1) * sr_t) + (T(n.u1) * sr_n)) * rho_div;
  r.u2 = ((T(t.u2) * sr_t) + (T(n.u2) * sr_n)) * rho_div;
  T const psi = ((psi_t * sr_t) + (psi_n * sr_n)) * rho_div;
  r.H = (T(t.H) * sr_t + T(n.H) * sr_n) * rho_div;
  r.gru = T(e.gamma - 1.0);
  r.q2 = sum_sq<DIM>(r.up * r.up, r.u1 * r.u1, r.u2 * r.u2);
  T const dup = T(t.up) - T(n.up), du1 = T(t.u1) - T(n.u1), du2 = T(t.u2) - T(n.u2);
  T const tmp = sum_sq<DIM>(dup * dup, du1 * du1, du2 * du2);
  // 0.5 rho_roe rho_div^2 = 0.5 w_t w_n
  T const jump = WEIGHTS ? T(0.5) * (sr_t * sr_n) * tmp
                         : T(0.5) * r.rho * (rho_div * rho_div) * tmp;
  T const p_over_rho =
      ((T(t.p) * T(t.one_rho)) * sr_t + (T(n.p) * T(n.one_rho)) * sr_n) * rho_div + jump;
  r.cc = psi + r.gru * p_over_rho;
  r.one_cc = quot(T(1), r.cc);
  r.c = tsqrt(r.cc);
  r.half_cc = T(0.5) * r.one_cc;
  return r;
}

// Row n of the left eigenvector matrix, indexed by conservative equation
// (eigendecomposition.h:316-359). Entries that are structurally zero are
// returned as 0 and skipped by the projection (adding 0*u leaves a sum unchanged).
template <int DIM, int DIR, typename T>
__device__ __forceinline__ void left_row(int n, Roe<T> const &r, T (&L)[DIM + 2]) {
  constexpr int NE = DIM + 2;
  constexpr int mP = MOMX + DIR;
  constexpr int m1 = MOMX + (DIM > 1 ? Minor<DIR>::m1 : 0);
  constexpr int m2 = MOMX + (DIM > 2 ? Minor<DIR>::m2 : 0);
#pragma unroll
  for (int l = 0; l < NE; ++l) L[l] = T(0);
  if (n == 0 || n == NE - 1) {
    T const sgn = n == 0 ? T(1) : T(-1);
    // 0.5/cc * (gru q^2 - gru H +/- (u +/- c) c)
    if (n == 0)
      L[MASS] = r.half_cc * (r.gru * r.q2 - r.gru * r.H + (r.up + r.c) * r.c);
    else
      L[MASS] = r.half_cc * (r.gru * r.q2 - r.gru * r.H - (r.up - r.c) * r.c);
    L[mP] = r.half_cc * (-r.up * r.gru - sgn * r.c);
    if (DIM > 1) L[m1] = r.half_cc * (-r.u1 * r.gru);
    if (DIM > 2) L[m2] = r.half_cc * (-r.u2 * r.gru);
    L[ENERGY] = r.half_cc * r.gru;
  } else if (n == DIM) {  // principal-momentum wave
    L[MASS] = r.one_cc * (r.H - r.q2);
    L[mP] = r.one_cc * r.up;
    if (DIM > 1) L[m1] = r.one_cc * r.u1;
    if (DIM > 2) L[m2] = r.one_cc * r.u2;
    L[ENERGY] = -r.one_cc;
  } else if (n == 1) {  // first minor momentum (DIM >= 2)
    L[MASS] = r.u1 * r.one_rho;
    L[m1] = -r.one_rho;
  } else {  // n == 2, second minor momentum (DIM == 3)
    L[MASS] = -r.u2 * r.one_rho;
    L[m2] = r.one_rho;
  }
}

// TransformToPhysicalSpace with generated right eigenvectors
// (eigendecomposition.h:144-165 and 366-409): linear waves summed first, then
// the nonlinear pair (u-c, u+c) added together.
template <int DIM, int DIR, typename T>
__device__ __forceinline__ void to_physical(Roe<T> const &r, T const (&ch)[DIM + 2],
                                            T (&out)[DIM + 2]) {
  constexpr int NE = DIM + 2;
  constexpr int EV = DIM;
  constexpr int mP = MOMX + DIR;
  constexpr int m1 = MOMX + (DIM > 1 ? Minor<DIR>::m1 : 0);
  constexpr int m2 = MOMX + (DIM > 2 ? Minor<DIR>::m2 : 0);
  // R[MASS][*] = (1, 0, 0, gru, 1)
  {
    T s = ch[EV] * r.gru;  // minor columns are zero
    out[MASS] = s + (ch[0] * T(1) + ch[NE - 1] * T(1));
  }
  // R[mP][*] = (u-c, 0, 0, gru*u, u+c)
  {
    T s = ch[EV] * (r.gru * r.up);
    out[mP] = s + (ch[0] * (r.up - r.c) + ch[NE - 1] * (r.up + r.c));
  }
  if constexpr (DIM > 1) {
    // R[m1][*] = (u1, -rho, 0, gru*u1, u1)
    T s = ch[1] * (-r.rho);
    s = s + ch[EV] * (r.gru * r.u1);
    out[m1] = s + (ch[0] * r.u1 + ch[NE - 1] * r.u1);
  }
  if constexpr (DIM > 2) {
    // R[m2][*] = (u2, 0, rho, gru*u2, u2)
    T s = ch[2] * r.rho;
    s = s + ch[EV] * (r.gru * r.u2);
    out[m2] = s + (ch[0] * r.u2 + ch[NE - 1] * r.u2);
  }
  // R[ENERGY][*] = (H - u c, -u1 rho, rho u2, gru H - c c, H + u c)
  {
    T s = T(0);
    if constexpr (DIM == 2) s = ch[1] * (-r.u1 * r.rho);
    if constexpr (DIM > 2) {
      // The two minor-wave terms are rounded as products before they are
      // added, so that the sum does not depend on which minor momentum is
      // numbered first: with the minor momenta exchanged (and their waves'
      // signs, as the characteristic variables then are) the bits are the
      // same. The strict build rounds every product anyway.
      T const t1 = rmul(ch[1], -r.u1 * r.rho);
      T const t2 = rmul(ch[2], r.rho * r.u2);
      s = t1 + t2;
    }
    s = s + ch[EV] * (r.gru * r.H - r.c * r.c);
    out[ENERGY] = s + (ch[0] * (r.H - r.up * r.c) + ch[NE - 1] * (r.H + r.up * r.c));
  }
}

// to_physical of both sides at once: ch[n] = (left, right) characteristic
// values; the same right-eigenvector entries, packed.
template <int DIM, int DIR>
__device__ __forceinline__ void to_physical_packed(Roe<float> const &r, float2 const (&ch)[DIM + 2],
                                                   float2 (&out)[DIM + 2]) {
  constexpr int NE = DIM + 2;
  constexpr int EV = DIM;
  constexpr int mP = MOMX + DIR;
  constexpr int m1 = MOMX + (DIM > 1 ? Minor<DIR>::m1 : 0);
  constexpr int m2 = MOMX + (DIM > 2 ? Minor<DIR>::m2 : 0);
  float2 const a = ch[0], z = ch[NE - 1], w = ch[EV];
  out[MASS] = fma2(w, dup2(r.gru), add2(a, z));
  out[mP] = fma2(w, dup2(r.gru * r.up), fma2(a, dup2(r.up - r.c), mul2(z, dup2(r.up + r.c))));
  if constexpr (DIM > 1)
    out[m1] = fma2(ch[1], dup2(-r.rho),
                   fma2(w, dup2(r.gru * r.u1), mul2(add2(a, z), dup2(r.u1))));
  if constexpr (DIM > 2)
    out[m2] = fma2(ch[2], dup2(r.rho),
                   fma2(w, dup2(r.gru * r.u2), mul2(add2(a, z), dup2(r.u2))));
  float2 s = fma2(w, dup2(r.gru * r.H - r.c * r.c),
                  fma2(a, dup2(r.H - r.up * r.c), mul2(z, dup2(r.H + r.up * r.c))));
  if constexpr (DIM == 2) s = fma2(ch[1], dup2(-r.u1 * r.rho), s);
  if constexpr (DIM > 2) {
    // the two minor-wave products rounded before they are added, as in
    // to_physical (the same bits with the minor momenta exchanged)
    s = add2(add2(mul2(ch[1], dup2(-r.u1 * r.rho)), mul2(ch[2], dup2(r.rho * r.u2))), s);
  }
  out[ENERGY] = s;
}

// ---- HLLC with Einfeldt signal speeds -------------------------------------
// CalculateSignalSpeed, Einfeldt (hll_signal_speed_calculator.h:77-101) and
// HllcRiemannSolver::SolveRiemannProblemImplementation (hllc_riemann_solver.h:52-198)
// one_rl, one_rr: 1/density of the two states as returned by inv()
template <int DIM, int DIR, typename T>
__device__ __forceinline__ void hllc(Eos const &e, T const (&cl)[DIM + 2], T const (&cr)[DIM + 2],
                                     T pres_l, T pres_r, T vel_l, T vel_r, T one_rl, T one_rr,
                                     T (&flux)[DIM + 2]) {
  constexpr int NE = DIM + 2;
  constexpr int mP = MOMX + DIR;
  T const c_l = eos_speed_of_sound<T>(e, cl[MASS], pres_l, one_rl);
  T const c_r = eos_speed_of_sound<T>(e, cr[MASS], pres_r, one_rr);
  T srl, srr, rho_div;
  if constexpr (ALP_FAST && sizeof(T) == 8) {
    // the Roe weights themselves (rho_div = 1): lambda = sqrt(rho_r / rho_l),
    // w_l = 1 / (1 + lambda), w_r = lambda w_l
    T const lambda = tsqrt(cr[MASS] * one_rl);
    srl = inv(T(1) + lambda);
    srr = lambda * srl;
    rho_div = T(1);
  } else {
    srl = tsqrt(cl[MASS]);
    srr = tsqrt(cr[MASS]);
    rho_div = quot(T(1), srl + srr);
  }
  T const u_roe = ((vel_l * srl) + (vel_r * srr)) * rho_div;
  T const c_e = tsqrt(((c_l * c_l * srl) + (c_r * c_r * srr)) * rho_div +
                     (T(0.5) * srl * srr * rho_div * rho_div) * (vel_r - vel_l) * (vel_r - vel_l));
  T const sls = dmin(u_roe - c_e, vel_l - c_l);
  T const srs = dmax(u_roe + c_e, vel_r + c_r);
  T const s_star = quot((pres_r - pres_l) + (cl[mP] * (sls - vel_l) - cr[mP] * (srs - vel_r)),
                        cl[MASS] * (sls - vel_l) - cr[MASS] * (srs - vel_r));
  if constexpr (ALP_FAST) {
    // The upwind star flux alone. Where the reference averages the two (S* = 0)
    // they are equal up to rounding: F*_L - F*_R = S* (U*_L - U*_R).
    bool const rs = s_star < T(0);
    T const rho = rs ? cr[MASS] : cl[MASS];
    T const mp = rs ? cr[mP] : cl[mP];
    T const E = rs ? cr[ENERGY] : cl[ENERGY];
    T const p = rs ? pres_r : pres_l;
    T const v = rs ? vel_r : vel_l;
    T const one_r = rs ? one_rr : one_rl;
    T const s = rs ? srs : sls;
    T const sc = rs ? dmax(srs, T(0)) : dmin(sls, T(0));
    T const chi = quot(s - v, s - s_star);
    T const rchi = rho * chi;
    flux[MASS] = mp + (sc * (rchi - rho));
    flux[mP] = ((mp * mp) * one_r + p) + (sc * (rchi * s_star - mp));
    T const es = rchi * (E * one_r + (s_star - v) * (s_star + quot(p, rho * (sc - v))));
    flux[ENERGY] = v * (E + p) + (sc * (es - E));
#pragma unroll
    for (int d = 0; d < DIM - 1; ++d) {
      int const mm = MOMX + (d == 0 ? Minor<DIR>::m1 : Minor<DIR>::m2);
      T const q = rs ? cr[mm] : cl[mm];
      flux[mm] = v * q + (sc * (chi * q - q));
    }
    return;
  }
  T const sl = dmin(sls, T(0));
  T const sr = dmax(srs, T(0));
  T const chi_l = quot(sls - vel_l, sls - s_star);
  T const chi_r = quot(srs - vel_r, srs - s_star);
  T const rchi_l = cl[MASS] * chi_l, rchi_r = cr[MASS] * chi_r;
  T const sg = T((T(0) < s_star) - (s_star < T(0)));
  T const wl = T(0.5) * (T(1) + sg), wr = T(0.5) * (T(1) - sg);
  // mass
  {
    T const fsl = cl[mP] + (sl * (rchi_l - cl[MASS]));
    T const fsr = cr[mP] + (sr * (rchi_r - cr[MASS]));
    flux[MASS] = wl * fsl + wr * fsr;
  }
  // principal momentum
  {
    T const fl = ((cl[mP] * cl[mP]) * one_rl) + pres_l;
    T const fr = ((cr[mP] * cr[mP]) * one_rr) + pres_r;
    T const fsl = fl + (sl * (rchi_l * s_star - cl[mP]));
    T const fsr = fr + (sr * (rchi_r * s_star - cr[mP]));
    flux[mP] = wl * fsl + wr * fsr;
  }
  // energy (the star-state pressure term uses the clamped speeds, :131-144)
  {
    T const el = rchi_l * (cl[ENERGY] * one_rl +
                           (s_star - vel_l) * (s_star + quot(pres_l, cl[MASS] * (sl - vel_l))));
    T const er = rchi_r * (cr[ENERGY] * one_rr +
                           (s_star - vel_r) * (s_star + quot(pres_r, cr[MASS] * (sr - vel_r))));
    T const fl = vel_l * (cl[ENERGY] + pres_l);
    T const fr = vel_r * (cr[ENERGY] + pres_r);
    T const fsl = fl + (sl * (el - cl[ENERGY]));
    T const fsr = fr + (sr * (er - cr[ENERGY]));
    flux[ENERGY] = wl * fsl + wr * fsr;
  }
  // minor momenta
#pragma unroll
  for (int d = 0; d < DIM - 1; ++d) {
    int const mm = MOMX + (d == 0 ? Minor<DIR>::m1 : Minor<DIR>::m2);
    T const fsl = vel_l * cl[mm] + (sl * (chi_l * cl[mm] - cl[mm]));
    T const fsr = vel_r * cr[mm] + (sr * (chi_r * cr[mm] - cr[mm]));
    flux[mm] = wl * fsl + wr * fsr;
  }
  (void)NE;
}

// HLLC for the FP32-flux form (same approximate Riemann solver as hllc():
// Einfeldt speeds, Toro star states, the reference's clamped-speed energy
// term). Wave speeds, the contact speed and the star-state increments
// q* - q are computed in float; the physical fluxes F(q) that carry the mean
// and their sum F + S (q* - q) are evaluated in double. Uses
// chi - 1 = (S* - u) / (S - S*), so no increment is formed by cancellation.
template <int DIM, int DIR>
__device__ __forceinline__ void hllc_mixed(Eos const &e, double const (&cl)[DIM + 2],
                                           double const (&cr)[DIM + 2], double pres_l,
                                           double pres_r, double vel_l, double vel_r,
                                           double one_rl, double one_rr, double (&flux)[DIM + 2]) {
  constexpr int mP = MOMX + DIR;
  float const g = float(e.gamma), B = float(e.B);
  float const rl = float(cl[MASS]), rr = float(cr[MASS]);
  float const ul = float(vel_l), ur = float(vel_r);
  float const cc_l = g * (float(pres_l) + B) * float(one_rl);
  float const cc_r = g * (float(pres_r) + B) * float(one_rr);
  float const c_l = tsqrt(cc_l), c_r = tsqrt(cc_r);
  float const srl = tsqrt(rl), srr = tsqrt(rr);
  float const rho_div = __fdividef(1.0f, srl + srr);
  float const u_roe = (ul * srl + ur * srr) * rho_div;
  float const c_e = tsqrt((cc_l * srl + cc_r * srr) * rho_div +
                          (0.5f * srl * srr * rho_div * rho_div) * (ur - ul) * (ur - ul));
  float const sls = dmin(u_roe - c_e, ul - c_l);
  float const srs = dmax(u_roe + c_e, ur + c_r);
  float const dpr = float(pres_r - pres_l);
  float const s_star = __fdividef(dpr + (rl * ul * (sls - ul) - rr * ur * (srs - ur)),
                                  rl * (sls - ul) - rr * (srs - ur));
  float const sl = dmin(sls, 0.0f), sr = dmax(srs, 0.0f);
  if constexpr (ALP_FAST) {
    // the upwind star flux alone (as in hllc())
    bool const rs = s_star < 0.0f;
    float const rho = rs ? rr : rl, u = rs ? ur : ul;
    float const s = rs ? srs : sls, sc = rs ? sr : sl;
    double const p = rs ? pres_r : pres_l, v = rs ? vel_r : vel_l;
    double const one_r = rs ? one_rr : one_rl;
    double const mp = rs ? cr[mP] : cl[mP], E = rs ? cr[ENERGY] : cl[ENERGY];
    float const dchi = __fdividef(s_star - u, s - s_star);  // chi - 1
    float dq[DIM + 2];
    double f[DIM + 2];
    dq[MASS] = rho * dchi;
    dq[mP] = rho * ((s_star - u) + dchi * s_star);
    dq[ENERGY] = float(E) * dchi + rho * (1.0f + dchi) * (s_star - u) *
                                       (s_star + __fdividef(float(p), rho * (sc - u)));
    f[MASS] = mp;
    f[mP] = mp * mp * one_r + p;
    f[ENERGY] = v * (E + p);
#pragma unroll
    for (int d = 0; d < DIM - 1; ++d) {
      int const mm = MOMX + (d == 0 ? Minor<DIR>::m1 : Minor<DIR>::m2);
      double const q = rs ? cr[mm] : cl[mm];
      dq[mm] = dchi * float(q);
      f[mm] = v * q;
    }
#pragma unroll
    for (int n = 0; n < DIM + 2; ++n) flux[n] = f[n] + double(sc * dq[n]);
    return;
  }
  float const dchi_l = __fdividef(s_star - ul, sls - s_star);  // chi_l - 1
  float const dchi_r = __fdividef(s_star - ur, srs - s_star);
  float const chi_l = 1.0f + dchi_l, chi_r = 1.0f + dchi_r;
  float const sg = float((0.0f < s_star) - (s_star < 0.0f));
  double const wl = 0.5 * (1.0 + sg), wr = 0.5 * (1.0 - sg);
  // star-state increments q* - q
  float dq_l[DIM + 2], dq_r[DIM + 2];
  dq_l[MASS] = rl * dchi_l;
  dq_r[MASS] = rr * dchi_r;
  dq_l[mP] = rl * ((s_star - ul) + dchi_l * s_star);
  dq_r[mP] = rr * ((s_star - ur) + dchi_r * s_star);
  dq_l[ENERGY] = float(cl[ENERGY]) * dchi_l +
                 rl * chi_l * (s_star - ul) *
                     (s_star + __fdividef(float(pres_l), rl * (sl - ul)));
  dq_r[ENERGY] = float(cr[ENERGY]) * dchi_r +
                 rr * chi_r * (s_star - ur) *
                     (s_star + __fdividef(float(pres_r), rr * (sr - ur)));
#pragma unroll
  for (int d = 0; d < DIM - 1; ++d) {
    int const mm = MOMX + (d == 0 ? Minor<DIR>::m1 : Minor<DIR>::m2);
    dq_l[mm] = dchi_l * float(cl[mm]);
    dq_r[mm] = dchi_r * float(cr[mm]);
  }
  // physical fluxes in double
  double fl[DIM + 2], fr[DIM + 2];
  fl[MASS] = cl[mP];
  fr[MASS] = cr[mP];
  fl[mP] = cl[mP] * cl[mP] * one_rl + pres_l;
  fr[mP] = cr[mP] * cr[mP] * one_rr + pres_r;
  fl[ENERGY] = vel_l * (cl[ENERGY] + pres_l);
  fr[ENERGY] = vel_r * (cr[ENERGY] + pres_r);
#pragma unroll
  for (int d = 0; d < DIM - 1; ++d) {
    int const mm = MOMX + (d == 0 ? Minor<DIR>::m1 : Minor<DIR>::m2);
    fl[mm] = vel_l * cl[mm];
    fr[mm] = vel_r * cr[mm];
  }
#pragma unroll
  for (int n = 0; n < DIM + 2; ++n)
    flux[n] = wl * (fl[n] + double(sl * dq_l[n])) + wr * (fr[n] + double(sr * dq_r[n]));
}

}  // namespace alp
