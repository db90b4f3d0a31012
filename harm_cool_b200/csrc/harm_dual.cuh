// Forward-mode dual numbers for the discrete adjoint's local Jacobians.
//
// Dual<N> carries a value and N directional derivatives.  The value part of
// every operation is the same IEEE double operation the plain step performs
// (the adjoint units are built with -fmad=false like the step), so a routine
// instantiated on Dual<N> reproduces the step's values bit for bit and its
// branches (limiters, floors, wave-speed selection) take the step's choices;
// the derivative parts are those of the branch taken.  Comparisons compare
// values only.  Operators are hidden friends, so unqualified sqrt/fabs on
// plain doubles still resolve to CUDA's.
#pragma once
#include <cmath>

namespace harm {

template <int N>
struct Dual {
  double v;
  double d[N];

  __device__ __forceinline__ Dual() {}
  __device__ __forceinline__ Dual(double x) : v(x)
  {
#pragma unroll
    for (int k = 0; k < N; k++) d[k] = 0.;
  }

  // the k-th input of a Jacobian column sweep: value x, derivative e_k
  __device__ __forceinline__ static Dual seed(double x, int k)
  {
    Dual r(x);
    if (k >= 0 && k < N) r.d[k] = 1.;
    return r;
  }

  friend __device__ __forceinline__ Dual operator+(const Dual &a, const Dual &b)
  {
    Dual r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] + b.d[k];
    return r;
  }
  friend __device__ __forceinline__ Dual operator-(const Dual &a, const Dual &b)
  {
    Dual r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] - b.d[k];
    return r;
  }
  friend __device__ __forceinline__ Dual operator*(const Dual &a, const Dual &b)
  {
    Dual r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
  }
  friend __device__ __forceinline__ Dual operator/(const Dual &a, const Dual &b)
  {
    Dual r;
    r.v = a.v / b.v;
    const double ib = 1. / b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
  }
  friend __device__ __forceinline__ Dual operator-(const Dual &a)
  {
    Dual r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = -a.d[k];
    return r;
  }

  // with plain doubles (constants and geometry)
  friend __device__ __forceinline__ Dual operator+(const Dual &a, double b)
  {
    Dual r = a;
    r.v = a.v + b;
    return r;
  }
  friend __device__ __forceinline__ Dual operator+(double a, const Dual &b)
  {
    Dual r = b;
    r.v = a + b.v;
    return r;
  }
  friend __device__ __forceinline__ Dual operator-(const Dual &a, double b)
  {
    Dual r = a;
    r.v = a.v - b;
    return r;
  }
  friend __device__ __forceinline__ Dual operator-(double a, const Dual &b)
  {
    Dual r;
    r.v = a - b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = -b.d[k];
    return r;
  }
  friend __device__ __forceinline__ Dual operator*(const Dual &a, double b)
  {
    Dual r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b;
    return r;
  }
  friend __device__ __forceinline__ Dual operator*(double a, const Dual &b)
  {
    Dual r;
    r.v = a * b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a * b.d[k];
    return r;
  }
  friend __device__ __forceinline__ Dual operator/(const Dual &a, double b)
  {
    Dual r;
    r.v = a.v / b;
    const double ib = 1. / b;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = a.d[k] * ib;
    return r;
  }
  friend __device__ __forceinline__ Dual operator/(double a, const Dual &b)
  {
    Dual r;
    r.v = a / b.v;
    const double f = -r.v / b.v;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = f * b.d[k];
    return r;
  }

  __device__ __forceinline__ Dual &operator+=(const Dual &b) { return *this = *this + b; }
  __device__ __forceinline__ Dual &operator-=(const Dual &b) { return *this = *this - b; }
  __device__ __forceinline__ Dual &operator*=(const Dual &b) { return *this = *this * b; }
  __device__ __forceinline__ Dual &operator/=(const Dual &b) { return *this = *this / b; }
  __device__ __forceinline__ Dual &operator+=(double b) { return *this = *this + b; }
  __device__ __forceinline__ Dual &operator-=(double b) { return *this = *this - b; }
  __device__ __forceinline__ Dual &operator*=(double b) { return *this = *this * b; }
  __device__ __forceinline__ Dual &operator/=(double b) { return *this = *this / b; }

  // sqrt: at a zero argument the derivative is taken as 0 (the one-sided
  // limit is unbounded; the step reaches sqrt(0) only through its clamps)
  friend __device__ __forceinline__ Dual sqrt(const Dual &a)
  {
    Dual r;
    r.v = sqrt(a.v);
    const double f = r.v > 0. ? 0.5 / r.v : 0.;
#pragma unroll
    for (int k = 0; k < N; k++) r.d[k] = f * a.d[k];
    return r;
  }
  friend __device__ __forceinline__ Dual fabs(const Dual &a)
  {
    return a.v < 0. ? -a : a;
  }

  friend __device__ __forceinline__ bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
  friend __device__ __forceinline__ bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
  friend __device__ __forceinline__ bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
  friend __device__ __forceinline__ bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }
  friend __device__ __forceinline__ bool operator<(const Dual &a, double b) { return a.v < b; }
  friend __device__ __forceinline__ bool operator>(const Dual &a, double b) { return a.v > b; }
  friend __device__ __forceinline__ bool operator<=(const Dual &a, double b) { return a.v <= b; }
  friend __device__ __forceinline__ bool operator>=(const Dual &a, double b) { return a.v >= b; }
  friend __device__ __forceinline__ bool operator<(double a, const Dual &b) { return a < b.v; }
  friend __device__ __forceinline__ bool operator>(double a, const Dual &b) { return a > b.v; }
  friend __device__ __forceinline__ bool operator<=(double a, const Dual &b) { return a <= b.v; }
  friend __device__ __forceinline__ bool operator>=(double a, const Dual &b) { return a >= b.v; }
};

}  // namespace harm
