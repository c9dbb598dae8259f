/* TEST INFRASTRUCTURE ONLY — operation counts of the oracle, never part of the
 * product path.
 *
 * Compiles the plain-C restatement (alpaca_oracle.c, which follows the
 * reference's operation order) as C++ with every `double` replaced by a scalar
 * that counts its floating-point operations. The counting scalar has the size
 * and layout of a double, so the entry points take the same buffers as
 * liboracle.so. The counts are the algorithmic operations of the reference
 * algorithm (what ALPACA's CPU code executes), used to state flops per face and
 * per cell-update and the FP64 compute ceiling of the path.
 *
 * Single-threaded: call the entry points with nthreads = 1.
 */
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>

namespace opcount {
long long add, mul, div, sqrt_, cmp, abs_, pow_, sin_;
}

struct cdouble {
  double v;
  cdouble() = default;
  constexpr cdouble(double x) : v(x) {}
  explicit operator double() const { return v; }
  explicit operator int() const { return (int)v; }
  cdouble &operator+=(cdouble o) { ++opcount::add; v += o.v; return *this; }
  cdouble &operator-=(cdouble o) { ++opcount::add; v -= o.v; return *this; }
  cdouble &operator*=(cdouble o) { ++opcount::mul; v *= o.v; return *this; }
  cdouble &operator/=(cdouble o) { ++opcount::div; v /= o.v; return *this; }
};
static_assert(sizeof(cdouble) == sizeof(double), "layout of a double");

inline cdouble operator+(cdouble a, cdouble b) { ++opcount::add; return a.v + b.v; }
inline cdouble operator-(cdouble a, cdouble b) { ++opcount::add; return a.v - b.v; }
inline cdouble operator*(cdouble a, cdouble b) { ++opcount::mul; return a.v * b.v; }
inline cdouble operator/(cdouble a, cdouble b) { ++opcount::div; return a.v / b.v; }
inline cdouble operator-(cdouble a) { return -a.v; }  // sign flip, no rounding
inline cdouble operator+(cdouble a) { return a; }
inline bool operator<(cdouble a, cdouble b) { ++opcount::cmp; return a.v < b.v; }
inline bool operator>(cdouble a, cdouble b) { ++opcount::cmp; return a.v > b.v; }
inline bool operator<=(cdouble a, cdouble b) { ++opcount::cmp; return a.v <= b.v; }
inline bool operator>=(cdouble a, cdouble b) { ++opcount::cmp; return a.v >= b.v; }
inline bool operator==(cdouble a, cdouble b) { ++opcount::cmp; return a.v == b.v; }
inline bool operator!=(cdouble a, cdouble b) { ++opcount::cmp; return a.v != b.v; }
inline cdouble sqrt(cdouble a) { ++opcount::sqrt_; return std::sqrt(a.v); }
inline cdouble fabs(cdouble a) { ++opcount::abs_; return std::fabs(a.v); }
inline cdouble pow(cdouble a, cdouble b) { ++opcount::pow_; return std::pow(a.v, b.v); }
inline cdouble sin(cdouble a) { ++opcount::sin_; return std::sin(a.v); }

#define double cdouble
#include "alpaca_oracle.c"
#undef double

extern "C" {

/* out[0..7] = additions/subtractions, multiplications, divisions, square
 * roots, comparisons, absolute values, powers, sines since the last reset. */
void oracle_op_counts(long long *out) {
  out[0] = opcount::add;
  out[1] = opcount::mul;
  out[2] = opcount::div;
  out[3] = opcount::sqrt_;
  out[4] = opcount::cmp;
  out[5] = opcount::abs_;
  out[6] = opcount::pow_;
  out[7] = opcount::sin_;
}

void oracle_op_reset(void) {
  opcount::add = opcount::mul = opcount::div = opcount::sqrt_ = opcount::cmp = opcount::abs_ = 0;
  opcount::pow_ = opcount::sin_ = 0;
}
}
