// Forward-mode derivative numbers for the Anand screening: a value and its derivative along one
// input direction. The screening kernel instantiated on Dual runs the same operations as on double
// and carries the derivative of every intermediate through them, iterations and all, so the
// result is the exact derivative of the discrete computation the screening performs (the quantity
// a finite difference of the screening converges to while no branch or iteration count changes).
// Branches and convergence tests compare values only.
#pragma once
#include <cmath>

namespace tmg {
// in a namespace of their own, so that the overloads below are found by argument-dependent lookup
// for Dual arguments and do not hide the standard functions for double arguments
namespace ad {

struct Dual {
  double v, d;
  __host__ __device__ Dual() : v(0), d(0) {}
  __host__ __device__ Dual(double x) : v(x), d(0) {}
  __host__ __device__ Dual(double x, double dx) : v(x), d(dx) {}
};

__device__ __forceinline__ double val(double x) { return x; }
__device__ __forceinline__ double val(const Dual& x) { return x.v; }

__device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual operator+(const Dual& a, double b) { return Dual(a.v + b, a.d); }
__device__ __forceinline__ Dual operator+(double a, const Dual& b) { return Dual(a + b.v, b.d); }
__device__ __forceinline__ Dual operator-(const Dual& a, double b) { return Dual(a.v - b, a.d); }
__device__ __forceinline__ Dual operator-(double a, const Dual& b) { return Dual(a - b.v, -b.d); }
__device__ __forceinline__ Dual operator*(const Dual& a, double b) { return Dual(a.v * b, a.d * b); }
__device__ __forceinline__ Dual operator*(double a, const Dual& b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator/(const Dual& a, double b) { return Dual(a.v / b, a.d / b); }
__device__ __forceinline__ Dual operator/(double a, const Dual& b) {
  const double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
__device__ __forceinline__ Dual& operator+=(Dual& a, const Dual& b) { a = a + b; return a; }
__device__ __forceinline__ Dual& operator-=(Dual& a, const Dual& b) { a = a - b; return a; }
__device__ __forceinline__ Dual& operator*=(Dual& a, const Dual& b) { a = a * b; return a; }

#define TM_DUAL_CMP(op)                                                                                      \
  __device__ __forceinline__ bool operator op(const Dual& a, const Dual& b) { return a.v op b.v; }          \
  __device__ __forceinline__ bool operator op(const Dual& a, double b) { return a.v op b; }                 \
  __device__ __forceinline__ bool operator op(double a, const Dual& b) { return a op b.v; }
TM_DUAL_CMP(<)
TM_DUAL_CMP(>)
TM_DUAL_CMP(<=)
TM_DUAL_CMP(>=)
TM_DUAL_CMP(==)
TM_DUAL_CMP(!=)
#undef TM_DUAL_CMP

__device__ __forceinline__ Dual fabs(const Dual& a) { return a.v < 0 ? -a : a; }
__device__ __forceinline__ Dual fmax(const Dual& a, const Dual& b) { return a.v >= b.v ? a : b; }
__device__ __forceinline__ Dual fmax(const Dual& a, double b) { return a.v >= b ? a : Dual(b); }
__device__ __forceinline__ Dual fmax(double a, const Dual& b) { return a >= b.v ? Dual(a) : b; }
__device__ __forceinline__ Dual fmin(const Dual& a, const Dual& b) { return a.v <= b.v ? a : b; }
__device__ __forceinline__ Dual fmin(const Dual& a, double b) { return a.v <= b ? a : Dual(b); }
__device__ __forceinline__ Dual fmin(double a, const Dual& b) { return a <= b.v ? Dual(a) : b; }
// derivatives of sqrt and pow at a zero argument would be infinite: a direction that does not move
// the argument contributes nothing there
__device__ __forceinline__ Dual sqrt(const Dual& a) {
  const double r = ::sqrt(a.v);
  return Dual(r, a.d == 0 ? 0.0 : 0.5 * a.d / r);
}
__device__ __forceinline__ Dual pow(const Dual& a, double p) {
  const double r = ::pow(a.v, p);
  return Dual(r, a.d == 0 ? 0.0 : p * ::pow(a.v, p - 1) * a.d);
}
__device__ __forceinline__ Dual sinh(const Dual& a) { return Dual(::sinh(a.v), ::cosh(a.v) * a.d); }
__device__ __forceinline__ Dual cosh(const Dual& a) { return Dual(::cosh(a.v), ::sinh(a.v) * a.d); }
__device__ __forceinline__ bool isfinite(const Dual& a) { return ::isfinite(a.v); }   // control flow follows values only
__device__ __forceinline__ double sgn(const Dual& v) { return v.v > 0 ? 1.0 : (v.v < 0 ? -1.0 : 0.0); }

}  // namespace ad
using ad::Dual;
}  // namespace tmg
