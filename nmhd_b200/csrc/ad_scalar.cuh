// Scalar types of the differentiated time step.
//
// The generic step (ad_cell.cuh) is written once over a scalar type T:
//   float          the FP32 step, operation for operation the production
//                  kernels (so an adjoint recomputation takes the same branches);
//   double         the FP64 step, the reference's Real = double build;
//   Dual<double>   forward-mode value + tangent: the FP64 tangent-linear step.
// Branches (limiter, Riemann fan region, upwind corner, min/max) are decided on
// values only, so a Dual run differentiates the branch actually taken.
//
// Everything here is __host__ __device__: the same code runs in the CUDA
// kernels and in the host-compiled check harness of the tests.
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define NMHD_HD __host__ __device__ __forceinline__
#else
#define NMHD_HD inline
#endif

namespace nmhd {
namespace ad {

// a*b + c rounded once.  The reverse sweeps accumulate their adjoints with it:
// they are checked against tangent-linear runs and differences to a
// tolerance, never bitwise against the reference, and a fused multiply-add is
// correctly rounded on the GPU and on the host alike, so the host build of the
// tests computes the same bits.  The forward arithmetic never uses it.
NMHD_HD float fmaa(float a, float b, float c) { return fmaf(a, b, c); }
NMHD_HD double fmaa(double a, double b, double c) { return fma(a, b, c); }

template <class R>
struct Dual {
  R v, d;
  NMHD_HD Dual() : v(0), d(0) {}
  NMHD_HD Dual(R x) : v(x), d(0) {}  // NOLINT: constants convert implicitly
  NMHD_HD Dual(R x, R dx) : v(x), d(dx) {}

  friend NMHD_HD Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
  friend NMHD_HD Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
  friend NMHD_HD Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
  friend NMHD_HD Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
  friend NMHD_HD Dual operator/(Dual a, Dual b) {
    const R q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
  }
  NMHD_HD Dual &operator+=(Dual b) { v += b.v; d += b.d; return *this; }
  NMHD_HD Dual &operator-=(Dual b) { v -= b.v; d -= b.d; return *this; }
  friend NMHD_HD bool operator<(Dual a, Dual b) { return a.v < b.v; }
  friend NMHD_HD bool operator>(Dual a, Dual b) { return a.v > b.v; }
  friend NMHD_HD bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
  friend NMHD_HD bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
};

// Base real of a scalar type, and the type the reference's double literals
// promote it to (float -> double; double and duals stay as they are).
template <class T> struct Traits { typedef T real; typedef T wide; };
template <> struct Traits<float> { typedef float real; typedef double wide; };
template <class R> struct Traits<Dual<R>> { typedef R real; typedef Dual<R> wide; };

NMHD_HD float val(float x) { return x; }
NMHD_HD double val(double x) { return x; }
template <class R> NMHD_HD R val(const Dual<R> &x) { return x.v; }

NMHD_HD float tan_of(float) { return 0.0f; }
NMHD_HD double tan_of(double) { return 0.0; }
template <class R> NMHD_HD R tan_of(const Dual<R> &x) { return x.d; }

// Conversions between scalar types (the tangent goes along).
template <class T> struct Conv;
template <> struct Conv<float> {
  NMHD_HD static float from(double x) { return (float)x; }
  NMHD_HD static float from(float x) { return x; }
};
template <> struct Conv<double> {
  NMHD_HD static double from(double x) { return x; }
  NMHD_HD static double from(float x) { return (double)x; }
};
template <class R> struct Conv<Dual<R>> {
  NMHD_HD static Dual<R> from(double x) { return Dual<R>((R)x); }
  NMHD_HD static Dual<R> from(float x) { return Dual<R>((R)x); }
  NMHD_HD static Dual<R> from(const Dual<R> &x) { return x; }
};
template <class T, class S> NMHD_HD T to(const S &x) { return Conv<T>::from(x); }

// Elementary functions.  sqrt'(0) and |x|'(0) are taken as 0 (the central
// difference of |x| at 0); min/max pick the first argument on a tie, as the
// library functions return it.
NMHD_HD float gsqrt(float x) { return sqrtf(x); }
NMHD_HD double gsqrt(double x) { return sqrt(x); }
template <class R> NMHD_HD Dual<R> gsqrt(const Dual<R> &a) {
  const R s = gsqrt(a.v);
  return Dual<R>(s, s > R(0) ? a.d / (s + s) : R(0));
}
NMHD_HD float gabs(float x) { return fabsf(x); }
NMHD_HD double gabs(double x) { return fabs(x); }
template <class R> NMHD_HD Dual<R> gabs(const Dual<R> &a) {
  return a.v > R(0) ? a : (a.v < R(0) ? -a : Dual<R>(R(0), R(0)));
}
NMHD_HD float gmin(float a, float b) { return fminf(a, b); }
NMHD_HD double gmin(double a, double b) { return fmin(a, b); }
template <class R> NMHD_HD Dual<R> gmin(const Dual<R> &a, const Dual<R> &b) { return b.v < a.v ? b : a; }
NMHD_HD float gmax(float a, float b) { return fmaxf(a, b); }
NMHD_HD double gmax(double a, double b) { return fmax(a, b); }
template <class R> NMHD_HD Dual<R> gmax(const Dual<R> &a, const Dual<R> &b) { return b.v > a.v ? b : a; }

}  // namespace ad
}  // namespace nmhd
